// SPDX-License-Identifier: GPL-3.0-or-later
// Host runtime of the dycore: handles (one or many domains), the device arena, the per-domain Dom
// tables, the halo refresh sets, the RK3 step as a sequence of batched launches (captured once into a
// CUDA graph and replayed), and the C ABI of include/cw_dycore.h (with cw_diagnostics of include/cw_output.h).
//
// The step order is CPPWRF's RK3::step (src/dyn/rk3.cpp:86-170): copy of the time-t state, then per RK
// stage rk_step_prep, rk_tendency (+ stage-1 diffusion and boundary relaxation), the acoustic loop,
// small_step_finish, scalar transport and calc_p_rho_phi; spec_bdy_final and set_w_surface at the end.
// Halos are refreshed where the reference refreshes them; refreshes with no kernel in between that
// reads the refreshed cells are merged into one launch.
#include <dlfcn.h>
#include <nccl.h>

#include "cw_step.cuh"

namespace {
thread_local std::string g_create_err;

template <class F>
int guarded(cw_handle* h, F f) {
  try {
    return f();
  } catch (const std::exception& e) {
    if (h) h->err = e.what();
    else g_create_err = e.what();
    return -1;
  }
}

size_t field_bytes(const cw_layout& L, int esz) { return size_t(L.total) * esz; }

template <class R>
V3<R> view3(char* base, const cw_layout& L) {
  return V3<R>{reinterpret_cast<R*>(base) + L.offset, int(L.sj), int(L.sk)};
}
template <class R>
VB<R> viewb(char* base, const cw_layout& L) {
  return VB<R>{reinterpret_cast<const R*>(base) + L.offset, int(L.si), int(L.sj), int(L.sk)};
}

// the device arena: every field of every member, vertical arrays, slabs
// some species of the member is advected positive-definite (the PD face-flux arrays are needed)
bool pd_any(const cw_options& o) {
  for (int n = 0; n < o.n_scalars; ++n)
    if ((n < o.n_moist ? o.moist_adv_opt : o.scalar_adv_opt) == 1) return true;
  return false;
}

// one member's allocation plan: byte offsets of every field, work field, scalar, vertical array and slab
struct Plan {
  std::vector<size_t> f, w, q1, qa, qb, qtf, qsc, qslab, qpd;
  size_t b64[3]{};
  size_t vert = 0;
  size_t slab[5]{};
  size_t total = 0;
};
Plan plan_member(Member& M) {
  Plan P;
  auto take = [&](size_t bytes) {
    const size_t off = P.total;
    P.total += align_up(bytes);
    return off;
  };
  M.L.resize(CW_Q_1);
  for (int id = 0; id < CW_Q_1; ++id) {
    M.L[id] = field_layout(M.g, M.o, id, M.pbox());
    P.f.push_back(take(field_bytes(M.L[id], M.esz)));
  }
  if (M.esz == 4)
    for (int x = 0; x < 3; ++x) P.b64[x] = take(field_bytes(M.L[kB64Fields[x]], 8));
  M.LW.resize(W_N);
  for (int w = 0; w < W_N; ++w) {
    const FieldKind k = work_kind(w);
    M.LW[w] = layout_make(M.g, k.stagger, k.rank, false, M.pbox());
    P.w.push_back(take(work_used(w, M.o) ? field_bytes(M.LW[w], M.esz) : 0));
  }
  M.Lq = layout_make(M.g, 'M', 3, false, M.pbox());
  for (int n = 0; n < M.o.n_scalars; ++n) {
    P.q1.push_back(take(field_bytes(M.Lq, M.esz)));
    P.qa.push_back(take(field_bytes(M.Lq, M.esz)));
    P.qb.push_back(take(field_bytes(M.Lq, M.esz)));
    P.qtf.push_back(take(field_bytes(M.Lq, M.esz)));
    P.qsc.push_back(take(field_bytes(M.Lq, M.esz)));
  }
  if (pd_any(M.o)) {
    M.Lpd[0] = layout_make(M.g, 'U', 3, false, M.pbox());
    M.Lpd[1] = layout_make(M.g, 'V', 3, false, M.pbox());
    M.Lpd[2] = layout_make(M.g, 'W', 3, false, M.pbox());
    for (int n = 0; n < M.o.n_scalars; ++n)
      for (int f = 0; f < 6; ++f) P.qpd.push_back(take(field_bytes(M.Lpd[f / 2], M.esz)));
  }
  P.vert = take(24 * size_t(M.g.nz + 2) * sizeof(double));
  for (int v = 0; v < 5; ++v) {
    size_t n = 0;
    if (M.o.lbc)
      for (int half = 0; half < 2; ++half)
        for (int sd = 0; sd < 4; ++sd) {
          M.slab_off[v][half * 4 + sd] = n;
          n += size_t(lbc_npos(M.g, v, sd)) * lbc_nk(M.g, v) * kLbcWidth;
        }
    P.slab[v] = M.o.lbc ? take(n * M.esz) : 0;
  }
  M.qslab_off.assign(M.o.n_scalars, {});
  M.q_have.assign(M.o.n_scalars, 0);
  for (int n = 0; n < M.o.n_scalars; ++n) {
    size_t cnt = 0;
    if (M.o.lbc)
      for (int half = 0; half < 2; ++half)
        for (int sd = 0; sd < 4; ++sd) {
          M.qslab_off[n][half * 4 + sd] = cnt;
          cnt += size_t(sd < 2 ? M.g.ny : M.g.nx) * M.g.nz * kLbcWidth;
        }
    P.qslab.push_back(M.o.lbc ? take(cnt * M.esz) : 0);
  }
  return P;
}

// the member's device arena (one cudaMalloc): every field, work field, scalar, vertical array and slab
void allocate_member(cw_handle* h, Member& M) {
  const Plan P = plan_member(M);
  CW_CUDA(cudaMalloc(&M.arena, P.total));
  M.arena_bytes = P.total;
  CW_CUDA(cudaMemsetAsync(M.arena, 0, P.total, h->stream));
  char* A = M.arena;
  M.base.clear();
  M.wbase.clear();
  M.q1.clear(); M.qa.clear(); M.qb.clear(); M.qtf.clear(); M.qsc.clear(); M.qslab.clear(); M.qpd.clear();
  for (size_t off : P.qpd) M.qpd.push_back(A + off);
  for (int id = 0; id < CW_Q_1; ++id) M.base.push_back(A + P.f[id]);
  for (int x = 0; x < 3; ++x) M.b64[x] = M.esz == 4 ? A + P.b64[x] : nullptr;
  for (int w = 0; w < W_N; ++w) M.wbase.push_back(A + P.w[w]);
  for (int n = 0; n < M.o.n_scalars; ++n) {
    M.q1.push_back(A + P.q1[n]);
    M.qa.push_back(A + P.qa[n]);
    M.qb.push_back(A + P.qb[n]);
    M.qtf.push_back(A + P.qtf[n]);
    M.qsc.push_back(A + P.qsc[n]);
    M.qslab.push_back(M.o.lbc ? A + P.qslab[n] : nullptr);
  }
  M.vert = reinterpret_cast<double*>(A + P.vert);
  for (int a = 0; a < 24; ++a) M.vert_off[a] = size_t(a) * (M.g.nz + 2);
  for (int v = 0; v < 5; ++v) M.slab[v] = M.o.lbc ? A + P.slab[v] : nullptr;
  // BaseState defaults: map factors and cosa = 1 (src/dyn/state.cpp:80-83)
  for (int id : {CW_MSFTX, CW_MSFTY, CW_MSFUX, CW_MSFUY, CW_MSFVX, CW_MSFVY, CW_MSFVX_INV, CW_COSA}) {
    const size_t n = size_t(M.L[id].total);
    if (M.esz == 8) {
      std::vector<double> one(n, 1.0);
      CW_CUDA(cudaMemcpyAsync(M.base[id], one.data(), n * 8, cudaMemcpyHostToDevice, h->stream));
      CW_CUDA(cudaStreamSynchronize(h->stream));
    } else {
      std::vector<float> one(n, 1.0f);
      CW_CUDA(cudaMemcpyAsync(M.base[id], one.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
      CW_CUDA(cudaStreamSynchronize(h->stream));
    }
  }
}

void allocate(cw_handle* h) {
  for (Member& M : h->m) allocate_member(h, M);
}

// vertical array slots in Member::vert
enum { VA_ZNU, VA_ZNW, VA_DNW, VA_DN, VA_RDNW, VA_RDN, VA_FNM, VA_FNP, VA_C1H, VA_C2H, VA_C1F, VA_C2F, VA_UB, VA_VB,
       VA_FCX, VA_GCX, VA_TB, VA_ZB, VA_C3H, VA_C4H, VA_C3F, VA_C4F };

template <class R>
Dom<R> make_dom(cw_handle* h, size_t mi, V3<R>* qtab_d, Slabs<R>* lbcq_d) {
  Member& M = h->m[mi];
  Dom<R> D{};
  const cw_grid& g = M.g;
  const cw_options& o = M.o;
  D.nx = g.nx; D.ny = g.ny; D.nz = g.nz; D.nyv = nys(g, 'V'); D.two_d = two_d(g); D.do_y = !two_d(g);
  const Box pb = M.patched ? M.patch : Box{0, g.nx, 0, g.ny};
  D.pi0 = pb.i0; D.pi1 = pb.i1; D.pj0 = pb.j0; D.pj1 = pb.j1;
  D.bc_x = g.bc_x; D.bc_y = g.bc_y;
  D.spec_x = flat_x(g); D.spec_y = flat_y(g) && !two_d(g);
  D.open_x = g.bc_x == CW_BC_OPEN; D.open_y = g.bc_y == CW_BC_OPEN && !two_d(g);
  D.sx = D.spec_x && !D.open_x; D.sy = D.spec_y && !D.open_y;
  D.lbc = o.lbc; D.flat = o.flat; D.n_moist = o.n_moist; D.n_scalars = o.n_scalars;
  D.diff_on = o.diff_opt == 1; D.top_lid = o.top_lid; D.w_damping = o.w_damping; D.n_sound = M.n_sound;
  D.moist_adv_opt = o.moist_adv_opt; D.scalar_adv_opt = o.scalar_adv_opt;
  D.mp_physics = o.mp_physics; D.mp_tend_lim = o.mp_tend_lim;
  D.damp_opt = o.damp_opt; D.zdamp = o.zdamp; D.dampcoef = o.dampcoef;
  D.diff_6th_opt = o.diff_6th_opt; D.diff_6th_factor = o.diff_6th_factor;
  D.dd_on = o.diff_opt == 1 || o.diff_6th_opt != 0 || o.damp_opt == 2;  // DiffusionConfig::on
  D.dt = g.dt; D.dx = g.dx; D.dy = g.dy; D.epssm = o.epssm; D.smdiv = o.smdiv; D.emdiv = o.emdiv; D.khdif = o.khdif; D.kvdif = o.kvdif;
  D.prandtl = 1.0 / o.pr_inv;
  D.hup = o.h_adv_order == 5 ? 1.0 : 0.0;
  D.vup = o.v_adv_order == 3 ? 1.0 : 0.0;
  D.w_crit_cfl = o.w_crit_cfl;
  D.dtbc = h->dtbc_d + mi;
  D.cfl = h->cfl_d + 6 * mi;
  D.status = h->status_d;
  D.cf1 = M.cf1; D.cf2 = M.cf2; D.cf3 = M.cf3; D.cfn = M.cfn; D.cfn1 = M.cfn1; D.rdx = M.rdx; D.rdy = M.rdy;
  const double* v = M.vert;
  auto va = [&](int a) { return v + M.vert_off[a]; };
  D.znu = va(VA_ZNU); D.znw = va(VA_ZNW); D.dnw = va(VA_DNW); D.dn = va(VA_DN); D.rdnw = va(VA_RDNW); D.rdn = va(VA_RDN);
  D.fnm = va(VA_FNM); D.fnp = va(VA_FNP); D.c1h = va(VA_C1H); D.c2h = va(VA_C2H); D.c1f = va(VA_C1F); D.c2f = va(VA_C2F);
  D.u_base = va(VA_UB); D.v_base = va(VA_VB); D.fcx = va(VA_FCX); D.gcx = va(VA_GCX);
  D.t_base = va(VA_TB); D.z_base = va(VA_ZB);
  D.c3h = va(VA_C3H); D.c4h = va(VA_C4H); D.c3f = va(VA_C3F); D.c4f = va(VA_C4F);
  D.hypsometric_opt = o.hypsometric_opt; D.p_top = g.p_top;
  auto f3 = [&](int id) { return view3<R>(M.base[id], M.L[id]); };
  auto fb = [&](int id) { return viewb<R>(M.base[id], M.L[id]); };
  auto w3 = [&](int w) { return view3<R>(M.wbase[w], M.LW[w]); };
  D.rainnc = f3(CW_RAINNC); D.rainncv = f3(CW_RAINNCV);
  D.u1 = f3(CW_U_1); D.u2 = f3(CW_U_2); D.v1 = f3(CW_V_1); D.v2 = f3(CW_V_2); D.w1 = f3(CW_W_1); D.w2 = f3(CW_W_2);
  D.t1 = f3(CW_T_1); D.t2 = f3(CW_T_2); D.ph1 = f3(CW_PH_1); D.ph2 = f3(CW_PH_2); D.mu1 = f3(CW_MU_1); D.mu2 = f3(CW_MU_2);
  D.p = f3(CW_P); D.al = f3(CW_AL); D.alt = f3(CW_ALT); D.php = f3(CW_PHP); D.ww = f3(CW_WW); D.mut = f3(CW_MUT);
  D.muu = f3(CW_MUU); D.muv = f3(CW_MUV); D.muts = f3(CW_MUTS); D.muus = f3(CW_MUUS); D.muvs = f3(CW_MUVS);
  D.ru = f3(CW_RU); D.rv = f3(CW_RV); D.rw = f3(CW_RW); D.ru_m = f3(CW_RU_M); D.rv_m = f3(CW_RV_M); D.ww_m = f3(CW_WW_M);
  D.cqu = f3(CW_CQU); D.cqv = f3(CW_CQV); D.cqw = f3(CW_CQW); D.hd = f3(CW_H_DIABATIC);
  D.ru_tend = f3(CW_RU_TEND); D.rv_tend = f3(CW_RV_TEND); D.rw_tend = f3(CW_RW_TEND); D.t_tend = f3(CW_T_TEND);
  D.ph_tend = f3(CW_PH_TEND); D.mu_tend = f3(CW_MU_TEND); D.ru_tendf = f3(CW_RU_TENDF); D.rv_tendf = f3(CW_RV_TENDF);
  D.rw_tendf = f3(CW_RW_TENDF); D.t_tendf = f3(CW_T_TENDF); D.ph_tendf = f3(CW_PH_TENDF);
  D.mub = fb(CW_MUB); D.pb = fb(CW_PB); D.alb = fb(CW_ALB); D.t_init = fb(CW_T_INIT); D.qv_base = fb(CW_QV_BASE);
  D.phb = fb(CW_PHB); D.ht = fb(CW_HT); D.msftx = fb(CW_MSFTX); D.msfty = fb(CW_MSFTY); D.msfux = fb(CW_MSFUX);
  D.msfuy = fb(CW_MSFUY); D.msfvx = fb(CW_MSFVX); D.msfvy = fb(CW_MSFVY); D.msfvx_inv = fb(CW_MSFVX_INV);
  D.f = fb(CW_F); D.e = fb(CW_E); D.sina = fb(CW_SINA); D.cosa = fb(CW_COSA); D.cor = o.coriolis != 0 || o.mapped != 0;
  auto f64 = [&](int x) { return viewb<double>(M.esz == 8 ? M.base[kB64Fields[x]] : M.b64[x], M.L[kB64Fields[x]]); };
  D.pb64 = f64(0); D.alb64 = f64(1); D.phb64 = f64(2);
  D.mapped = o.mapped != 0;
  D.u_save = w3(W_U_SAVE); D.v_save = w3(W_V_SAVE); D.w_save = w3(W_W_SAVE); D.t_save = w3(W_T_SAVE);
  D.ph_save = w3(W_PH_SAVE); D.ww1 = w3(W_WW1); D.c2a = w3(W_C2A); D.pm1 = w3(W_PM1); D.t_2save = w3(W_T_2SAVE);
  D.a = w3(W_A); D.alpha = w3(W_ALPHA); D.gamma = w3(W_GAMMA); D.mu_save = w3(W_MU_SAVE); D.mudf = w3(W_MUDF);
  D.muave = w3(W_MUAVE); D.w_rhs = w3(W_W_RHS); D.t2a = w3(W_T2A);
  if (xk_fields(o)) { D.xkmh = w3(W_XKMH); D.xkhh = w3(W_XKHH); }
  D.km_opt = o.km_opt; D.xk_field = xk_fields(o) && o.diff_opt == 1;
  const int ns = o.n_scalars;
  D.q1 = qtab_d; D.q2 = qtab_d + ns; D.qn = qtab_d + 2 * ns; D.qtf = qtab_d + 3 * ns; D.qscale = qtab_d + 4 * ns;
  D.qpd = qtab_d + 5 * ns;
  for (int var = 0; var < 5; ++var) {
    Slabs<R>& s = D.lbc_var[var];
    s.nk = lbc_nk(g, var);
    s.have = o.lbc;
    for (int sd = 0; sd < 4; ++sd) {
      s.npos[sd] = lbc_npos(g, var, sd);
      s.v[sd] = M.slab[var] ? reinterpret_cast<const R*>(M.slab[var]) + M.slab_off[var][sd] : nullptr;
      s.t[sd] = M.slab[var] ? reinterpret_cast<const R*>(M.slab[var]) + M.slab_off[var][4 + sd] : nullptr;
    }
  }
  D.lbc_q = lbcq_d;
  return D;
}

// member m's first block of each index range and block shape, and each range's block total
template <class SET>
std::array<std::array<int, kNumShapes>, kNumKinds> block_starts(cw_handle* h, size_t m0, int n, SET set) {
  std::array<std::array<int, kNumShapes>, kNumKinds> tot{};
  for (int kind = 0; kind < kNumKinds; ++kind)
    for (int sh = 0; sh < kNumShapes; ++sh) {
      long long b = 0;
      for (int m = 0; m < n; ++m) {
        const Member& M = h->m[m0 + size_t(m)];
        set(kind, sh, m, int(b));
        const Box pb = M.patched ? M.patch : Box{0, M.g.nx, 0, M.g.ny};
        b += blocks_of(range_of(kind, M.g.nx, M.g.ny, M.g.nz, nys(M.g, 'V'), pb.i0, pb.i1, pb.j0, pb.j1), kind, sh);
      }
      if (b >= (1ll << 31)) throw std::runtime_error("a batch launch of more than 2^31 blocks");
      set(kind, sh, n, int(b));
      tot[size_t(kind)][size_t(sh)] = int(b);
    }
  return tot;
}
// a single domain: its descriptor in the launch parameter
template <class R>
void build_packs(cw_handle* h, const std::vector<Dom<R>>& doms, Packs<R, 1>& ps) {
  ps.p.clear();
  ps.blocks.clear();
  if (doms.size() != 1) return;
  Pack<R, 1> P{};
  P.n = 1;
  P.d[0] = doms[0];
  ps.blocks.push_back(block_starts(h, 0, 1, [&](int kind, int sh, int m, int b) { P.start_[kind][sh][m] = b; }));
  ps.p.push_back(P);
}
// a batch: every member's descriptor in device memory and the block starts in the launch parameter, one pack (one
// launch per kernel)
template <class R>
void build_packs(cw_handle* h, const std::vector<Dom<R>>& doms, DevTables<R>& T) {
  Packs<R, 0>& ps = T.many;
  ps.p.clear();
  ps.blocks.clear();
  const size_t nm = doms.size();
  if (nm <= 1) return;
  auto P = std::make_unique<Pack<R, 0>>();
  ps.blocks.push_back(block_starts(h, 0, int(nm), [&](int kind, int sh, int m, int b) { P->start_[kind][sh][m] = b; }));
  CW_CUDA(cudaMalloc(&T.doms_d, nm * sizeof(Dom<R>)));
  CW_CUDA(cudaMemcpyAsync(T.doms_d, doms.data(), nm * sizeof(Dom<R>), cudaMemcpyHostToDevice, h->stream));
  CW_CUDA(cudaStreamSynchronize(h->stream));  // the host vector goes out of scope
  P->d = T.doms_d;
  P->n = int(nm);
  ps.p.push_back(*P);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver library)
using EncodeTiled = decltype(&cuTensorMapEncodeTiled);
EncodeTiled encode_tiled() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return EncodeTiled(nullptr);
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}
// the tensor map of one scalar buffer for k_q_march: the allocation as (pitch, rows, levels), a box of one plane of
// a tile with its halo; false where the layout does not allow it (2-D, narrower than the box, unaligned)
template <class R>
bool encode_q_map(CUtensorMap* out, const char* base, const cw_layout& L) {
  const EncodeTiled enc = encode_tiled();
  constexpr int W = QPlanes<R>::W, H = QPlanes<R>::H;
  const int64_t rows = L.wj1 - L.wj0;
  if (!enc || L.sj <= 0 || L.sj < W || rows < H || L.nz < 1) return false;
  if ((reinterpret_cast<uintptr_t>(base) % 16) != 0 || (L.sj * int64_t(sizeof(R))) % 16 != 0 ||
      (L.sk * int64_t(sizeof(R))) % 16 != 0 || L.sk != L.sj * rows)
    return false;
  const cuuint64_t dims[3] = {cuuint64_t(L.sj), cuuint64_t(rows), cuuint64_t(L.nz)};
  const cuuint64_t strides[2] = {cuuint64_t(L.sj) * sizeof(R), cuuint64_t(L.sk) * sizeof(R)};
  const cuuint32_t box[3] = {cuuint32_t(W), cuuint32_t(H), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(out, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                         const_cast<char*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}
// member M's maps (one per species) for k_q_march, false if any cannot be made. Element (i, j, k) of a scalar
// buffer is at offset + i + j sj + k sk with offset = x0 + y0 sj, x0 = 5 - wi0 (a row's 8-element lead before its
// halo of 3), y0 = -wj0: the map coordinates of i = 0, j = 0. The tiles start at i = pi0 + 32 b, so the x of a
// tile's first staged column, x0 + pi0 - 4 + 32 b = 4 + 32 b, is 16-byte aligned.
template <class R>
bool make_q_maps(const Member& M, std::vector<QMap>& out) {
  if (two_d(M.g) || M.o.n_scalars == 0) return false;
  const cw_layout& L = M.Lq;
  const int x0 = 5 - L.wi0, y0 = -L.wj0;
  const int pi0 = M.patched ? M.patch.i0 : 0;
  if (L.offset != int64_t(x0) + int64_t(y0) * L.sj) return false;  // the layout's lead as assumed above
  if ((int64_t(x0 + pi0 - 4) * int64_t(sizeof(R))) % 16 != 0) return false;
  for (int n = 0; n < M.o.n_scalars; ++n) {
    QMap q{};
    if (!encode_q_map<R>(&q.a, M.qa[size_t(n)], L) || !encode_q_map<R>(&q.b, M.qb[size_t(n)], L)) return false;
    q.pa = view3<R>(M.qa[size_t(n)], L).p;
    q.x0 = x0;
    q.y0 = y0;
    out.push_back(q);
  }
  return true;
}

template <class R>
void upload_tables(cw_handle* h, DevTables<R>& T) {
  const size_t nm = h->m.size();
  if (nm == 0) return;
  if (!h->dtbc_d) CW_CUDA(cudaMalloc(&h->dtbc_d, nm * sizeof(double)));
  if (!h->cfl_d) {
    CW_CUDA(cudaMalloc(&h->cfl_d, 6 * nm * sizeof(unsigned long long)));
    CW_CUDA(cudaMemsetAsync(h->cfl_d, 0, 6 * nm * sizeof(unsigned long long), h->stream));
  }
  size_t nq = 0;
  for (const Member& M : h->m) nq += size_t(M.o.n_scalars);
  if (!T.qtab && nq) CW_CUDA(cudaMalloc(&T.qtab, kQTab * nq * sizeof(V3<R>)));
  if (!T.lbcq && nq) CW_CUDA(cudaMalloc(&T.lbcq, nq * sizeof(Slabs<R>)));
  if (!h->status_d) {
    CW_CUDA(cudaMalloc(&h->status_d, sizeof(unsigned)));
    CW_CUDA(cudaMemsetAsync(h->status_d, 0, sizeof(unsigned), h->stream));
  }
  // the TMA-staged scalar update where every member allows it (3-D, wide enough for a tile's planes)
  std::vector<QMap> qmaps;
  bool q_tma = nq > 0;
  for (const Member& M : h->m)
    if (q_tma && M.o.n_scalars > 0) q_tma = make_q_maps<R>(M, qmaps);
  h->q_tma = q_tma;
  if (q_tma && !T.qmap) CW_CUDA(cudaMalloc(&T.qmap, qmaps.size() * sizeof(QMap)));
  std::vector<Dom<R>> doms(nm);
  std::vector<V3<R>> qtab(kQTab * nq);
  std::vector<Slabs<R>> lbcq(nq);
  size_t q0 = 0;
  for (size_t mi = 0; mi < nm; ++mi) {
    Member& M = h->m[mi];
    const int ns = M.o.n_scalars;
    doms[mi] = make_dom<R>(h, mi, T.qtab ? T.qtab + kQTab * q0 : nullptr, T.lbcq ? T.lbcq + q0 : nullptr);
    doms[mi].qmap = q_tma ? T.qmap + q0 : nullptr;
    for (int n = 0; n < ns; ++n) {
      char* q2 = M.q_parity ? M.qb[n] : M.qa[n];
      char* qn = M.q_parity ? M.qa[n] : M.qb[n];
      qtab[kQTab * q0 + n] = view3<R>(M.q1[n], M.Lq);
      qtab[kQTab * q0 + ns + n] = view3<R>(q2, M.Lq);
      qtab[kQTab * q0 + 2 * ns + n] = view3<R>(qn, M.Lq);
      qtab[kQTab * q0 + 3 * ns + n] = view3<R>(M.qtf[n], M.Lq);
      qtab[kQTab * q0 + 4 * ns + n] = view3<R>(M.qsc[n], M.Lq);
      if (!M.qpd.empty())
        for (int f = 0; f < 6; ++f) qtab[kQTab * q0 + 5 * ns + 6 * n + f] = view3<R>(M.qpd[6 * size_t(n) + f], M.Lpd[f / 2]);
      Slabs<R>& s = lbcq[q0 + n];
      s.nk = M.g.nz;
      s.have = M.o.lbc && M.q_have[n];
      for (int sd = 0; sd < 4; ++sd) {
        s.npos[sd] = sd < 2 ? M.g.ny : M.g.nx;
        s.v[sd] = M.qslab[n] ? reinterpret_cast<const R*>(M.qslab[n]) + M.qslab_off[n][sd] : nullptr;
        s.t[sd] = M.qslab[n] ? reinterpret_cast<const R*>(M.qslab[n]) + M.qslab_off[n][4 + sd] : nullptr;
      }
    }
    q0 += size_t(ns);
  }
  build_packs(h, doms, T.one);
  build_packs(h, doms, T);
  std::vector<double> dtbc(nm);
  for (size_t mi = 0; mi < nm; ++mi) dtbc[mi] = h->m[mi].dtbc;
  CW_CUDA(cudaMemcpyAsync(h->dtbc_d, dtbc.data(), nm * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  if (nq) {
    CW_CUDA(cudaMemcpyAsync(T.qtab, qtab.data(), qtab.size() * sizeof(V3<R>), cudaMemcpyHostToDevice, h->stream));
    CW_CUDA(cudaMemcpyAsync(T.lbcq, lbcq.data(), lbcq.size() * sizeof(Slabs<R>), cudaMemcpyHostToDevice, h->stream));
  }
  if (q_tma) CW_CUDA(cudaMemcpyAsync(T.qmap, qmaps.data(), qmaps.size() * sizeof(QMap), cudaMemcpyHostToDevice, h->stream));
  CW_CUDA(cudaStreamSynchronize(h->stream));
}

void upload_tables(cw_handle* h) {
  if (h->precision == CW_FP64) upload_tables<double>(h, h->t64);
  else upload_tables<float>(h, h->t32);
}

void size_column_blocks(cw_handle* h) {
  h->nzmax = 0;
  for (const Member& M : h->m) h->nzmax = std::max(h->nzmax, M.g.nz);
  h->cb_level_bytes = size_t(h->nzmax + 2) * CX * sizeof(double);
}

// ---- halo sets
enum HaloParity { HP_DEFAULT, HP_EVEN, HP_ODDFACE_X, HP_ODD_Y };
struct HaloItem {
  char* base;        // allocation (nullptr: indirect)
  void* ind;         // indirect view address
  cw_layout L;
  int parity;
  int fid;           // the field: its id, or FID_W + work field, FID_Q2 / FID_Q1 / FID_QSC + species
};
enum : int { FID_W = 1000, FID_Q2 = 2000, FID_Q1 = 3000, FID_QSC = 4000 };

HaloField halo_field(const Member& M, const HaloItem& it) {
  HaloField f{};
  const cw_layout& L = it.L;
  f.p = it.base ? it.base + size_t(L.offset) * M.esz : nullptr;
  f.ind = it.ind;
  f.sj = int(L.sj);
  f.sk = int(L.sk);
  f.lnx = L.nx;
  f.lny = L.ny;
  f.nk = L.nz;
  f.wi0 = L.wi0; f.wi1 = L.wi1; f.wj0 = L.wj0; f.wj1 = L.wj1;
  f.gnx = M.g.nx;
  f.gny = M.g.ny;
  f.periodic_x = M.g.bc_x == CW_BC_PERIODIC;
  f.periodic_y = M.g.bc_y == CW_BC_PERIODIC;
  f.flat_x = flat_x(M.g);
  f.flat_y = flat_y(M.g);
  f.two_d = two_d(M.g);
  f.face_x = L.stagger == 'U';
  f.face_y = L.stagger == 'V';
  const bool three = L.rank == 3;
  switch (it.parity) {
    case HP_DEFAULT: f.odd_x = three && L.stagger == 'U'; f.odd_y = three && L.stagger == 'V'; break;
    case HP_ODDFACE_X: f.odd_x = 1; f.oddface_x = 1; break;
    case HP_ODD_Y: f.odd_y = 1; break;
    default: break;
  }
  f.is_float = M.esz == 4;
  f.xj0 = L.wj0 > 0 ? L.wj0 : 0;
  f.xj1 = L.wj1 < L.ny ? L.wj1 : L.ny;
  f.ncell_x = (long long)(f.face_x ? 8 : 6) * (f.xj1 - f.xj0) * L.nz;
  f.ncell = f.ncell_x + (f.two_d ? 0 : (long long)(f.face_y ? 8 : 6) * (L.wi1 - L.wi0) * L.nz);
  return f;
}

void finish_haloset(cw_handle*, HaloSetHost& s) {
  s.small.clear();
  s.large.clear();
  if (s.f.size() <= size_t(kHaloSmall)) chunk_fields(s.f, s.small);
  else chunk_fields(s.f, s.large);
}
// the points of a field of staggering s ('U', 'V', else mass / W) that a patch owns: its cells' (the faces nx / ny
// at the domain's east / north edge)
Box owned_box(const Member& M, char s) {
  const Box& p = M.patch;
  return Box{p.i0, (s == 'U' && p.i1 == M.g.nx) ? M.g.nx + 1 : p.i1, p.j0,
             (s == 'V' && p.j1 == M.g.ny && !two_d(M.g)) ? M.g.ny + 1 : p.j1};
}
// the rectangle of a field's window (layout L of some patch) that patch t owns, all levels
bool exchange_rect(const cw_layout& L, const Member& t, XchgBox& x) {
  if (L.uniform) return false;
  const Box o = owned_box(t, L.stagger);
  x = XchgBox{};
  x.i0 = std::max(L.wi0, o.i0);
  x.i1 = std::min(L.wi1, o.i1);
  x.j0 = std::max(L.wj0, o.j0);
  x.j1 = std::min(L.wj1, o.j1);
  if (x.i0 >= x.i1 || x.j0 >= x.j1) return false;
  x.nk = L.nz;
  x.ncell = (long long)(x.i1 - x.i0) * (x.j1 - x.j0) * x.nk;
  return true;
}
// the source side of a box: the owner's field (element (0, 0, 0) or its table entry)
void box_source(XchgBox& x, const Member& t, const HaloItem& b) {
  x.src = b.base ? b.base + size_t(b.L.offset) * t.esz : nullptr;
  x.src_ind = b.ind;
  x.ssj = int(b.L.sj);
  x.ssk = int(b.L.sk);
  x.is_float = t.esz == 4;
}
// the destination side: the receiving patch's field
void box_dest(XchgBox& x, const Member& me, const HaloItem& a) {
  x.dst = a.base ? a.base + size_t(a.L.offset) * me.esz : nullptr;
  x.dst_ind = a.ind;
  x.dsj = int(a.L.sj);
  x.dsk = int(a.L.sk);
  x.is_float = me.esz == 4;
}

// one field of a fill point: its set (the fill point), the field, and whether the fill only refreshes the points of
// the neighbouring patches (no boundary fill)
struct FillItem {
  int set;
  HaloItem it;
  bool xonly;
};
// The fields of every fill point of member M, in one order (the same for every patch of a decomposed domain, whose
// patches share their options). qt: the member's scalar table in device memory, null for a patch of another rank
// (its items carry layouts only).
template <class R>
std::vector<FillItem> fill_items(const Member& M, V3<R>* qt) {
  std::vector<FillItem> v;
  const int ns = M.o.n_scalars;
  auto at = [](const std::vector<char*>& b, size_t k) -> char* { return k < b.size() ? b[k] : nullptr; };
  auto F = [&](int id, int par = HP_DEFAULT) { return HaloItem{at(M.base, size_t(id)), nullptr, M.L[id], par, id}; };
  auto W = [&](int w, int par = HP_DEFAULT) {
    return HaloItem{at(M.wbase, size_t(w)), nullptr, M.LW[w], par, FID_W + w};
  };
  auto Q2 = [&](int n) { return HaloItem{nullptr, qt ? qt + ns + n : nullptr, M.Lq, HP_DEFAULT, FID_Q2 + n}; };
  auto add = [&](int set, std::initializer_list<HaloItem> its) {
    for (const HaloItem& it : its) v.push_back(FillItem{set, it, false});
  };
  auto exchange_only = [&](int set, const HaloItem& it) { v.push_back(FillItem{set, it, true}); };
  const bool spec = specified(M.g);
  add(cw_handle::H_MU1, {F(CW_MU_1)});
  if (xk_fields(M.o)) add(cw_handle::H_XK, {W(W_XKMH), W(W_XKHH)});  // DiffusionDriver::prepare's fill
  add(cw_handle::H_PREP0, {F(CW_U_2), F(CW_V_2), F(CW_W_2), F(CW_T_2), F(CW_PH_2), F(CW_P), F(CW_AL)});
  if (!spec) add(cw_handle::H_PREP0, {F(CW_MU_2)});
  else {  // tiles: the neighbours' points that spec_bdy_final changed (large_step.cpp:705; the scalars' too)
    exchange_only(cw_handle::H_PREP0, F(CW_MU_2));
    for (int n = 0; n < ns; ++n) exchange_only(cw_handle::H_PREP0, Q2(n));
  }
  add(cw_handle::H_PREP1, {F(CW_MUT), F(CW_RU), F(CW_RV), F(CW_RW), F(CW_ALT), F(CW_PHP), F(CW_MUU, HP_ODDFACE_X),
                           F(CW_MUV, HP_ODD_Y), F(CW_WW)});
  add(cw_handle::H_SS0, {F(CW_U_2), F(CW_V_2), F(CW_PH_2), W(W_T_SAVE), W(W_U_SAVE), W(W_V_SAVE), F(CW_MU_2),
                         F(CW_MUTS), F(CW_P), F(CW_AL)});
  add(cw_handle::H_UV, {F(CW_U_2)});
  if (!two_d(M.g)) add(cw_handle::H_UV, {F(CW_V_2)});
  add(cw_handle::H_AC, {F(CW_MU_2), W(W_MUDF), F(CW_MUTS), F(CW_PH_2), F(CW_P), F(CW_AL)});
  add(cw_handle::H_POST, {F(CW_MUTS), F(CW_RU_M), F(CW_RV_M), F(CW_WW_M)});
  add(cw_handle::H_FIN, {F(CW_U_2), F(CW_V_2), F(CW_W_2), F(CW_T_2), F(CW_PH_2), F(CW_WW), F(CW_MU_2), F(CW_P), F(CW_AL)});
  for (int n = 0; n < ns; ++n) {
    add(cw_handle::H_Q1PD, {HaloItem{at(M.q1, size_t(n)), nullptr, M.Lq, HP_DEFAULT, FID_Q1 + n}});
    add(cw_handle::H_SCPD, {HaloItem{at(M.qsc, size_t(n)), nullptr, M.Lq, HP_DEFAULT, FID_QSC + n}});
    add(cw_handle::H_Q2, {Q2(n)});
  }
  add(cw_handle::H_END_P, {F(CW_P), F(CW_AL)});
  if (M.o.mp_physics != 0) {  // PhysicsCoupling::step's halos (physics_coupling.cpp:452-456), then calc_p_rho_phi's
    add(cw_handle::H_MP, {F(CW_T_2), F(CW_H_DIABATIC)});
    for (int n = 0; n < M.o.n_moist; ++n) add(cw_handle::H_MP, {Q2(n)});
    add(cw_handle::H_MP_P, {F(CW_P), F(CW_AL)});
  }
  add(cw_handle::H_WS0, {F(CW_U_2), F(CW_V_2)});
  add(cw_handle::H_WS1, {F(CW_W_2)});
  return v;
}

// patch t's rank in a decomposed domain over ranks
inline int rank_of(const cw_handle* h, int t) { return t % h->nranks; }

// (device: false for a plan made without a device, cw_decomp_plan: no exchange buffer)
template <class R>
void build_halosets_t(cw_handle* h, DevTables<R>& T, bool device = true) {
  const bool dec = h->decomp_px > 0;
  const int np = dec ? h->decomp_px * h->decomp_py : 0;
  std::vector<std::vector<FillItem>> items(dec ? size_t(np) : 0);  // a decomposed domain: by patch number
  std::vector<const Member*> pat(items.size(), nullptr);
  std::vector<char> local(items.size(), 0);
  size_t q0 = 0;
  for (size_t mi = 0; mi < h->m.size(); ++mi) {
    Member& M = h->m[mi];
    std::vector<FillItem> v = fill_items<R>(M, T.qtab ? T.qtab + kQTab * q0 : nullptr);
    for (const FillItem& fi : v)
      if (!fi.xonly) h->hs[fi.set].f.push_back(halo_field(M, fi.it));
    if (dec) {
      const size_t t = size_t(M.tid);
      pat[t] = &M;
      local[t] = 1;
      items[t] = std::move(v);
    }
    q0 += size_t(M.o.n_scalars);
  }
  for (const Member& M : h->remote) {
    pat[size_t(M.tid)] = &M;
    items[size_t(M.tid)] = fill_items<R>(M, nullptr);
  }
  // every patch receives, at each fill point, the points of its window that the others own: a box between two
  // patches of one rank is copied directly, a box between ranks is packed by the owner's rank, transferred and
  // unpacked by the receiver's (both ranks list it in the same order: receiving patch, owning patch, field)
  size_t send_cap = 0, recv_cap = 0;
  for (int me = 0; me < np; ++me)
    for (int t = 0; t < np; ++t) {
      if (t == me || (!local[size_t(me)] && !local[size_t(t)])) continue;
      if (!pat[size_t(me)] || !pat[size_t(t)]) throw std::runtime_error("decomposition: a patch is missing");
      const std::vector<FillItem>& A = items[size_t(me)];
      const std::vector<FillItem>& B = items[size_t(t)];
      if (A.size() != B.size()) throw std::runtime_error("decomposition: patches differ");
      const bool cross = h->loopback ? rank_of(h, me) != rank_of(h, t) : !(local[size_t(me)] && local[size_t(t)]);
      for (size_t k = 0; k < A.size(); ++k) {
        XchgBox x;
        if (!exchange_rect(A[k].it.L, *pat[size_t(t)], x)) continue;
        if (!cross) {
          box_source(x, *pat[size_t(t)], B[k].it);
          box_dest(x, *pat[size_t(me)], A[k].it);
          h->hs[A[k].set].x.push_back(x);
          continue;
        }
        RBox r{};
        r.me = me;
        r.t = t;
        r.fid = A[k].it.fid;
        r.src_rank = rank_of(h, t);
        r.dst_rank = rank_of(h, me);
        r.has_send = local[size_t(t)] != 0;
        r.has_recv = local[size_t(me)] != 0;
        r.send = r.recv = x;
        if (r.has_send) {
          box_source(r.send, *pat[size_t(t)], B[k].it);
          send_cap += size_t(x.ncell);
        }
        if (r.has_recv) {
          box_dest(r.recv, *pat[size_t(me)], A[k].it);
          recv_cap += size_t(x.ncell);
        }
        h->hs[A[k].set].r.push_back(r);
      }
    }
  if (device && send_cap + recv_cap > 0) {  // every fill point's boxes fit (a fill point is a union of sets)
    const size_t esz = h->m.empty() ? 8 : size_t(h->m[0].esz);
    CW_CUDA(cudaMalloc(&h->xbuf, (send_cap + recv_cap) * esz));
    h->xsend_cap = send_cap;
    h->xrecv_cap = recv_cap;
  }
  for (int s = 0; s < cw_handle::H_N; ++s) finish_haloset(h, h->hs[s]);
}

void build_copies(cw_handle* h) {
  // step start: u_1 = u_2, ... (whole allocations, src/dyn/rk3.cpp:95-99); q_1 = q_2 read through the table
  size_t q0 = 0;
  for (Member& M : h->m) {
    const int pairs[6][2] = {{CW_U_1, CW_U_2}, {CW_V_1, CW_V_2}, {CW_W_1, CW_W_2}, {CW_T_1, CW_T_2}, {CW_PH_1, CW_PH_2}, {CW_MU_1, CW_MU_2}};
    for (auto& p : pairs)
      h->copies.push_back(CopyDesc{M.base[p[0]], M.base[p[1]], nullptr, M.L[p[0]].total, M.esz == 4, 0});
    const int ns = M.o.n_scalars;
    for (int n = 0; n < ns; ++n) {
      // src through the device table entry q2[n].p (the element (0,0,0) pointer): offset back to the allocation
      const void* const* ind = nullptr;
      if (h->precision == CW_FP64) ind = reinterpret_cast<const void* const*>(&(h->t64.qtab + kQTab * q0 + ns + n)->p);
      else ind = reinterpret_cast<const void* const*>(&(h->t32.qtab + kQTab * q0 + ns + n)->p);
      CopyDesc c{M.q1[n], nullptr, ind, M.Lq.total, M.esz == 4, M.Lq.offset};
      h->copies.push_back(c);
    }
    h->zeros.push_back(CopyDesc{M.wbase[W_MUDF], nullptr, nullptr, M.LW[W_MUDF].total, M.esz == 4, 0});
    q0 += size_t(ns);
  }
  auto up = [&](std::vector<CopyDesc>& v, CopyDesc*& d, long long*& sd, long long& total) {
    if (v.empty()) return;
    std::vector<long long> st(v.size() + 1, 0);
    for (size_t n = 0; n < v.size(); ++n) st[n + 1] = st[n] + v[n].n;
    total = st.back();
    CW_CUDA(cudaMalloc(&d, v.size() * sizeof(CopyDesc)));
    CW_CUDA(cudaMalloc(&sd, st.size() * sizeof(long long)));
    CW_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(CopyDesc), cudaMemcpyHostToDevice));
    CW_CUDA(cudaMemcpy(sd, st.data(), st.size() * sizeof(long long), cudaMemcpyHostToDevice));
  };
  up(h->copies, h->copies_d, h->copies_start_d, h->copies_total);
  up(h->zeros, h->zeros_d, h->zeros_start_d, h->zeros_total);
}

// ---- the step
// the FP64 form's kernels are instantiated in this file (compiled without FMA contraction); the mixed form's in
// cw_step_mixed.cu, compiled with its own floating-point options
void enqueue(cw_handle* h, Launcher& L) {
  if (h->precision == CW_FP64) enqueue_t<double>(h, L, h->t64);
  else L.count += enqueue_mixed(h, L.plan);
}

void invalidate_graph(cw_handle* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->gexec = nullptr;
  h->graph = nullptr;
  h->graph_ok = false;
}

// one eager step with every tunable point kernel in block shape `shape`, each launch timed by events
void tune_step(cw_handle* h, int shape) {
  auto saved = std::move(h->prof_ev);
  h->prof_ev.clear();
  const bool was = h->profiling;
  h->profiling = true;
  h->tuning_shape = shape;
  Launcher L{h};
  try {
    enqueue(h, L);
  } catch (...) {
    h->profiling = was;
    h->tuning_shape = -1;
    throw;
  }
  h->profiling = was;
  h->tuning_shape = -1;
  CW_CUDA(cudaStreamSynchronize(h->stream));
  for (auto& [name, ev] : h->prof_ev) {
    float ms = 0;
    CW_CUDA(cudaEventElapsedTime(&ms, ev.first, ev.second));
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
    auto it = std::find_if(h->tune_ms.begin(), h->tune_ms.end(), [&](const auto& e) { return e.first == name; });
    if (it == h->tune_ms.end()) {
      h->tune_ms.push_back({name, {}});
      it = h->tune_ms.end() - 1;
    }
    it->second[size_t(shape)] += ms;
  }
  h->prof_ev = std::move(saved);
  h->launches_last += L.count;
}

// after the tuning steps: every kernel keeps its fastest shape (the lowest on a tie); the scalar update is the
// faster of the point kernel k_q_update and the TMA-staged k_q_march, each in its fastest shape (each was timed in
// one round of steps, in every shape)
void finish_tuning(cw_handle* h) {
  h->shape_choice.clear();
  float best_update = -1, best_march = -1;
  for (const auto& [name, ms] : h->tune_ms) {
    int best = 0;
    for (int sh = 1; sh < kNumShapes; ++sh)
      if (ms[size_t(sh)] < ms[size_t(best)]) best = sh;
    h->shape_choice.push_back({name, best});
    if (name == "k_q_update") best_update = ms[size_t(best)];
    if (name == "k_q_march") best_march = ms[size_t(best)];
  }
  h->q_march = best_march >= 0 && best_update >= 0 && best_march < best_update;
  h->tuned = true;
  invalidate_graph(h);
}

void run_steps(cw_handle* h, int nsteps) {
  h->launches_last = 0;
  if (h->m.empty()) return;
  // tuning steps advance the state like any other step: kTuneRounds rounds of one step per shape, the order reversed
  // in every other round (a drift over the steps weighs on every shape alike); each kernel's times summed over them
  while (h->autotune && !h->tuned && nsteps > 0) {
    const int s = h->tune_steps_done, idx = s % kNumShapes;
    tune_step(h, (s / kNumShapes) % 2 == 0 ? idx : kNumShapes - 1 - idx);
    for (Member& M : h->m) {
      if (M.o.lbc) M.dtbc += M.g.dt;
      if (M.o.n_scalars > 0) M.q_parity ^= 1;
    }
    --nsteps;
    if (++h->tune_steps_done == kNumShapes * kTuneRounds) finish_tuning(h);
  }
  if (nsteps == 0) return;
  if (h->use_graph && !h->graph_ok) {
    if (h->m.size() > 1 || h->decomp_px > 0) {  // a batch's halo tables are device allocations: made before the capture
      Launcher P{h};
      P.plan = true;
      enqueue(h, P);
    }
    Launcher L{h};
    CW_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue(h, L);
    } catch (...) {
      cudaGraph_t g;
      cudaStreamEndCapture(h->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CW_CUDA(cudaStreamEndCapture(h->stream, &h->graph));
    CW_CUDA(cudaGraphInstantiate(&h->gexec, h->graph, 0));
    h->graph_ok = true;
    h->launches_step = L.count;
  }
  for (int s = 0; s < nsteps; ++s) {
    if (h->use_graph) {
      CW_CUDA(cudaGraphLaunch(h->gexec, h->stream));
      h->launches_last += h->launches_step;
    } else {
      Launcher L{h};
      enqueue(h, L);
      h->launches_step = L.count;
      h->launches_last += L.count;
    }
    for (Member& M : h->m) {
      if (M.o.lbc) M.dtbc += M.g.dt;
      if (M.o.n_scalars > 0) M.q_parity ^= 1;  // three swaps per step
    }
  }
}

Member make_member(const cw_grid& g, const cw_options& o) {
  if (const char* why = unsupported(g, o)) throw std::runtime_error(why);
  Member M;
  M.g = g;
  M.o = o;
  M.n_sound = sound_steps(g, o);
  M.esz = o.precision == CW_MIXED ? 4 : 8;
  return M;
}

// the handle-level device tables (scalar tables, boundary clocks, halo and copy descriptors), freed before
// they are rebuilt for a new set of members
void free_tables(cw_handle* h) {
  for (auto& hs : h->hs) hs = HaloSetHost{};
  for (auto& kv : h->halo_tabs) {
    cudaFree(kv.second.f);
    cudaFree(kv.second.start);
    cudaFree(kv.second.x);
    cudaFree(kv.second.xstart);
    cudaFree(kv.second.pk);
    cudaFree(kv.second.pkstart);
  }
  h->halo_tabs.clear();
  cudaFree(h->xbuf);
  h->xbuf = nullptr;
  h->xsend_cap = h->xrecv_cap = 0;
  cudaFree(h->copies_d);
  cudaFree(h->copies_start_d);
  cudaFree(h->zeros_d);
  cudaFree(h->zeros_start_d);
  h->copies.clear();
  h->zeros.clear();
  h->copies_d = h->zeros_d = nullptr;
  h->copies_start_d = h->zeros_start_d = nullptr;
  h->copies_total = h->zeros_total = 0;
  cudaFree(h->dtbc_d);
  h->dtbc_d = nullptr;
  cudaFree(h->cfl_d);  // member count changes with the tables: reallocated (zeroed) with them
  h->cfl_d = nullptr;
  cudaFree(h->t64.qtab);
  cudaFree(h->t64.lbcq);
  cudaFree(h->t64.doms_d);
  cudaFree(h->t64.qmap);
  cudaFree(h->t32.qtab);
  cudaFree(h->t32.lbcq);
  cudaFree(h->t32.doms_d);
  cudaFree(h->t32.qmap);
  h->q_tma = false;
  h->t64 = DevTables<double>{};
  h->t32 = DevTables<float>{};
}

void build_tables(cw_handle* h) {
  upload_tables(h);
  size_column_blocks(h);
  if (h->precision == CW_FP64) build_halosets_t<double>(h, h->t64);
  else build_halosets_t<float>(h, h->t32);
  build_copies(h);
}

// a new set of members: every handle-level table is rebuilt and the step is captured again
void rebuild(cw_handle* h) {
  CW_CUDA(cudaStreamSynchronize(h->stream));
  invalidate_graph(h);
  free_tables(h);
  build_tables(h);
}

void setup(cw_handle* h) {
  CW_CUDA(cudaGetDevice(&h->device));
  allocate(h);
  build_tables(h);
}

// locate a field: allocation and layout
struct Loc {
  char* base;
  cw_layout L;
  int esz;
  char* b64 = nullptr;  // the mixed form's double copy of the field (PB, ALB, PHB), written with it
};
Loc locate(cw_handle* h, int mi, int field, int n) {
  if (mi < 0 || mi >= int(h->m.size())) throw std::runtime_error("member index out of range");
  Member& M = h->m[mi];
  if (field >= 0 && field < CW_Q_1) {
    const int x = b64_slot(field);
    return Loc{M.base[field], M.L[field], M.esz, x >= 0 ? M.b64[x] : nullptr};
  }
  if (n < 0 || n >= M.o.n_scalars) throw std::runtime_error("scalar index out of range");
  if (field == CW_Q_1) return Loc{M.q1[n], M.Lq, M.esz};
  if (field == CW_Q_2) return Loc{M.q_parity ? M.qb[n] : M.qa[n], M.Lq, M.esz};
  if (field == CW_Q_TENDF) return Loc{M.qtf[n], M.Lq, M.esz};
  throw std::runtime_error("unknown field id");
}

__global__ void k_widen(const float* __restrict__ src, double* __restrict__ dst, unsigned n) {
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) dst[t] = double(src[t]);
}
__global__ void k_narrow(const double* __restrict__ src, float* __restrict__ dst, unsigned n) {
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) dst[t] = float(src[t]);
}

// the handle's double staging buffer of at least n elements (FP32 fields are converted on the device)
double* staging(cw_handle* h, size_t n) {
  if (h->staging_n < n) {
    CW_CUDA(cudaStreamSynchronize(h->stream));
    cudaFree(h->staging);
    h->staging = nullptr;
    h->staging_n = 0;
    CW_CUDA(cudaMalloc(&h->staging, n * sizeof(double)));
    h->staging_n = n;
  }
  return h->staging;
}

void copy_in(cw_handle* h, const Loc& l, const double* host, size_t count) {
  if (count != size_t(l.L.total)) throw std::runtime_error("count != layout.total");
  if (count >= (size_t(1) << 32)) throw std::runtime_error("field too large");
  if (l.esz == 8) {
    CW_CUDA(cudaMemcpyAsync(l.base, host, count * 8, cudaMemcpyHostToDevice, h->stream));
  } else {  // doubles to the staging buffer, narrowed to float on the device (round to nearest)
    double* st = staging(h, count);
    CW_CUDA(cudaMemcpyAsync(st, host, count * 8, cudaMemcpyHostToDevice, h->stream));
    const unsigned n = unsigned(count), blocks = std::min(4096u, (n + 255u) / 256u);
    k_narrow<<<blocks, 256, 0, h->stream>>>(st, reinterpret_cast<float*>(l.base), n);
    CW_CUDA(cudaGetLastError());
    if (l.b64) CW_CUDA(cudaMemcpyAsync(l.b64, st, count * 8, cudaMemcpyDeviceToDevice, h->stream));
  }
}
void copy_out(cw_handle* h, const Loc& l, double* host, size_t count) {
  if (count != size_t(l.L.total)) throw std::runtime_error("count != layout.total");
  if (count >= (size_t(1) << 32)) throw std::runtime_error("field too large");
  if (l.esz == 8) {
    CW_CUDA(cudaMemcpyAsync(host, l.base, count * 8, cudaMemcpyDeviceToHost, h->stream));
  } else {  // widened to double on the device, then copied
    double* st = staging(h, count);
    const unsigned n = unsigned(count), blocks = std::min(4096u, (n + 255u) / 256u);
    k_widen<<<blocks, 256, 0, h->stream>>>(reinterpret_cast<const float*>(l.base), st, n);
    CW_CUDA(cudaGetLastError());
    CW_CUDA(cudaMemcpyAsync(host, st, count * 8, cudaMemcpyDeviceToHost, h->stream));
  }
  CW_CUDA(cudaStreamSynchronize(h->stream));
}

// ---- non-finite detection (the reference's run.check_nonfinite_every_step)
// the smallest key (field slot, k, j, i) of a non-finite interior value of one field
template <class T>
__global__ void k_nonfinite(const T* __restrict__ p, int sj, int sk, int nx, int ny, int nz, unsigned long long base,
                            unsigned long long* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)nx * ny * nz;
  if (t >= n) return;
  const int i = int(t % nx), j = int((t / nx) % ny), k = int(t / ((long long)nx * ny));
  const T v = p[i + j * (long long)sj + k * (long long)sk];
  if (!isfinite(v)) atomicMin(out, base + (unsigned long long)t);
}

// cw_diagnostics of member mi: the per-level partials on the device, folded over the levels in order here
// (Reducer::run's host loop, src/core/backend.hpp:857-859; Diagnostics::compute, src/dyn/diagnostics.cpp:56-80)
template <class R>
void diagnostics_t(cw_handle* h, int mi, DevTables<R>& T, cw_diag* out) {
  size_t q0 = 0;
  for (int m = 0; m < mi; ++m) q0 += size_t(h->m[size_t(m)].o.n_scalars);
  const Dom<R> D = make_dom<R>(h, size_t(mi), T.qtab ? T.qtab + kQTab * q0 : nullptr, T.lbcq ? T.lbcq + q0 : nullptr);
  const Member& M = h->m[size_t(mi)];
  const int nz = M.g.nz, K1 = nz + 1;
  const size_t need = size_t(DG_NPART) * size_t(K1);
  if (h->diag_part_n < need) {
    cudaFree(h->diag_part);
    h->diag_part = nullptr;
    h->diag_part_n = 0;
    CW_CUDA(cudaMalloc(&h->diag_part, need * sizeof(double)));
    h->diag_part_n = need;
  }
  constexpr double r_d = 287.0, r_v = 461.6, cp = 7.0 * r_d / 2.0;  // src/core/constants.hpp:5-14
  const DiagConst c{r_v / r_d, r_d / cp, cp - r_d};
  k_diag<R><<<dim3(unsigned(K1), 4), kDiagThreads, 0, h->stream>>>(D, c, h->diag_part);
  CW_CUDA(cudaGetLastError());
  std::vector<double> hp(need);
  CW_CUDA(cudaMemcpyAsync(hp.data(), h->diag_part, need * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CW_CUDA(cudaStreamSynchronize(h->stream));
  auto fold_max = [&](int q, int nk) {
    double a = -1e308;
    for (int k = 0; k < nk; ++k) a = hp[size_t(q) * K1 + k] > a ? hp[size_t(q) * K1 + k] : a;
    return a;
  };
  auto fold_sum = [&](int q, int nk) {
    double a = 0.0;
    for (int k = 0; k < nk; ++k) a = a + hp[size_t(q) * K1 + k];
    return a;
  };
  const double area = M.g.dx * (two_d(M.g) ? 1.0 : M.g.dy) / 9.81;
  out->max_abs_u = fold_max(DG_MAX_U, nz);
  out->max_abs_v = fold_max(DG_MAX_V, nz);
  out->max_abs_w = fold_max(DG_MAX_W, nz + 1);
  out->max_th_pert = fold_max(DG_MAX_THP, nz);
  out->min_th_pert = -fold_max(DG_MAX_THM, nz);
  out->dry_mass = area * fold_sum(DG_SUM_MASS, 1);
  out->theta_mass = area * fold_sum(DG_SUM_THETA, nz);
  out->total_energy = area * fold_sum(DG_SUM_ENERGY, nz);
  const double mq = fold_max(DG_MAX_Q, nz);
  out->max_abs_q = 0.0 < mq ? mq : 0.0;
}

// a decomposed domain's handle on this process: its patches (every patch when loopback or nranks == 1), the other
// ranks' patches as layouts; no device work
std::unique_ptr<cw_handle> decomp_handle(const cw_grid* g, const cw_options* o, int px, int py, int rank, int nranks,
                                         bool loopback) {
  if (!g || !o) throw std::runtime_error("null argument");
  if (const char* why = decomp_unsupported(*g, px, py)) throw std::runtime_error(why);
  if (nranks < 1 || nranks > px * py || rank < 0 || rank >= nranks)
    throw std::runtime_error("decomposition: 0 <= rank < nranks <= px * py");
  auto h = std::make_unique<cw_handle>();
  h->precision = o->precision;
  h->decomp_px = px;
  h->decomp_py = py;
  h->rank = rank;
  h->nranks = nranks;
  h->loopback = loopback && nranks > 1;
  for (int t = 0; t < px * py; ++t) {
    Member M = make_member(*g, *o);
    M.patched = true;
    M.patch = patch_box(*g, px, py, t);
    M.tid = t;
    if (h->loopback || t % nranks == rank) {
      h->m.push_back(std::move(M));
    } else {
      plan_member(M);  // the layouts of its fields
      h->remote.push_back(std::move(M));
    }
  }
  return h;
}

// NCCL, loaded when the first decomposed domain over ranks is made (libnccl.so.2: the one the process has loaded
// already, if any); nothing else needs it
struct NcclApi {
  bool ok = false;
  std::string err;
  decltype(&ncclGetUniqueId) GetUniqueId = nullptr;
  decltype(&ncclCommInitRank) CommInitRank = nullptr;
  decltype(&ncclCommDestroy) CommDestroy = nullptr;
  decltype(&ncclSend) Send = nullptr;
  decltype(&ncclRecv) Recv = nullptr;
  decltype(&ncclGroupStart) GroupStart = nullptr;
  decltype(&ncclGroupEnd) GroupEnd = nullptr;
  decltype(&ncclGetErrorString) GetErrorString = nullptr;
};
const NcclApi& nccl_api() {
  static const NcclApi api = [] {
    NcclApi a;
    void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) {
      const char* e = dlerror();
      a.err = std::string("NCCL: ") + (e ? e : "libnccl.so.2 not found");
      return a;
    }
    bool ok = true;
    auto sym = [&](auto& f, const char* name) {
      f = reinterpret_cast<std::remove_reference_t<decltype(f)>>(dlsym(lib, name));
      ok &= f != nullptr;
    };
    sym(a.GetUniqueId, "ncclGetUniqueId");
    sym(a.CommInitRank, "ncclCommInitRank");
    sym(a.CommDestroy, "ncclCommDestroy");
    sym(a.Send, "ncclSend");
    sym(a.Recv, "ncclRecv");
    sym(a.GroupStart, "ncclGroupStart");
    sym(a.GroupEnd, "ncclGroupEnd");
    sym(a.GetErrorString, "ncclGetErrorString");
    a.ok = ok;
    if (!ok) a.err = "NCCL: a symbol is missing from libnccl.so.2";
    return a;
  }();
  return api;
}
void nccl_check(const NcclApi& N, ncclResult_t r, const char* what) {
  if (r != ncclSuccess) throw std::runtime_error(std::string(what) + ": " + N.GetErrorString(r));
}

// ---- several fields in one call (cw_upload_fields / cw_upload_windows and the downloads)
// The rows of a field's window: `rows` rows of `width` points at stride `pitch`, the first at element `first` of the
// allocation (the levels' windows follow each other at the same stride: sk = sj (wj1 - wj0), or sj = 0 in 2-D with
// sk the row stride). Otherwise (horizontally uniform storage) the whole allocation as one row.
struct WinRows {
  size_t first, width, pitch, rows;
};
WinRows window_rows(const cw_layout& L) {
  const size_t w = size_t(L.wi1 - L.wi0), nj = size_t(L.wj1 - L.wj0), nk = size_t(L.rank == 3 ? L.nz : 1);
  if (!L.uniform && L.sj > 0 && (L.rank != 3 || size_t(L.sk) == size_t(L.sj) * nj))
    return WinRows{size_t(L.offset + L.wi0 + int64_t(L.wj0) * L.sj), w, size_t(L.sj), nj * nk};
  if (!L.uniform && L.sj == 0 && L.rank == 3 && nj == 1 && L.sk > 0)
    return WinRows{size_t(L.offset + L.wi0 + int64_t(L.wj0) * L.sj), w, size_t(L.sk), nk};
  return WinRows{0, size_t(L.total), size_t(L.total), 1};
}
// one field's copy: the whole allocation, or its window's rows (window)
void copy_rows(cw_handle* h, char* dst, const char* src, const cw_layout& L, bool window, cudaMemcpyKind kind) {
  if (!window) {
    CW_CUDA(cudaMemcpyAsync(dst, src, size_t(L.total) * 8, kind, h->stream));
    return;
  }
  const WinRows r = window_rows(L);
  CW_CUDA(cudaMemcpy2DAsync(dst + r.first * 8, r.pitch * 8, src + r.first * 8, r.pitch * 8, r.width * 8, r.rows, kind,
                            h->stream));
}
std::vector<Loc> locate_all(cw_handle* h, int mi, int nf, const int* fields, const int* ns, const void* const* host,
                            const size_t* counts, size_t& staged) {
  if (!h || nf < 0 || (nf > 0 && (!fields || !ns || !host || !counts))) throw std::runtime_error("null argument");
  std::vector<Loc> locs;
  staged = 0;
  for (int f = 0; f < nf; ++f) {
    if (!host[f]) throw std::runtime_error("null host buffer");
    locs.push_back(locate(h, mi, fields[f], ns[f]));
    if (counts[f] != size_t(locs.back().L.total)) throw std::runtime_error("count != layout.total");
    if (counts[f] >= (size_t(1) << 32)) throw std::runtime_error("field too large");
    if (locs.back().esz != 8) staged += counts[f];
  }
  return locs;
}
// FP64 fields copy directly; FP32 (mixed) fields go through one staging region per field (the staging buffer sized
// for all of them first, so that no reallocation happens between the copies; with window copies it is zeroed first,
// so that the narrowed row padding holds zeros)
void upload_fields(cw_handle* h, int mi, int nf, const int* fields, const int* ns, const double* const* host,
                   const size_t* counts, bool window) {
  size_t staged = 0;
  const std::vector<Loc> locs =
      locate_all(h, mi, nf, fields, ns, reinterpret_cast<const void* const*>(host), counts, staged);
  double* st = staged ? staging(h, staged) : nullptr;
  if (st && window) CW_CUDA(cudaMemsetAsync(st, 0, staged * sizeof(double), h->stream));
  for (int f = 0; f < nf; ++f) {
    const Loc& l = locs[size_t(f)];
    if (l.esz == 8) {
      copy_rows(h, l.base, reinterpret_cast<const char*>(host[f]), l.L, window, cudaMemcpyHostToDevice);
    } else {
      copy_rows(h, reinterpret_cast<char*>(st), reinterpret_cast<const char*>(host[f]), l.L, window,
                cudaMemcpyHostToDevice);
      const unsigned n = unsigned(counts[f]), blocks = std::min(4096u, (n + 255u) / 256u);
      k_narrow<<<blocks, 256, 0, h->stream>>>(st, reinterpret_cast<float*>(l.base), n);
      CW_CUDA(cudaGetLastError());
      if (l.b64) CW_CUDA(cudaMemcpyAsync(l.b64, st, counts[f] * 8, cudaMemcpyDeviceToDevice, h->stream));
      st += counts[f];
    }
  }
}
void download_fields(cw_handle* h, int mi, int nf, const int* fields, const int* ns, double* const* host,
                     const size_t* counts, bool window) {
  size_t staged = 0;
  const std::vector<Loc> locs =
      locate_all(h, mi, nf, fields, ns, reinterpret_cast<const void* const*>(host), counts, staged);
  double* st = staged ? staging(h, staged) : nullptr;
  for (int f = 0; f < nf; ++f) {
    const Loc& l = locs[size_t(f)];
    if (l.esz == 8) {
      copy_rows(h, reinterpret_cast<char*>(host[f]), l.base, l.L, window, cudaMemcpyDeviceToHost);
    } else {
      const unsigned n = unsigned(counts[f]), blocks = std::min(4096u, (n + 255u) / 256u);
      k_widen<<<blocks, 256, 0, h->stream>>>(reinterpret_cast<const float*>(l.base), st, n);
      CW_CUDA(cudaGetLastError());
      copy_rows(h, reinterpret_cast<char*>(host[f]), reinterpret_cast<const char*>(st), l.L, window,
                cudaMemcpyDeviceToHost);
      st += counts[f];
    }
  }
  CW_CUDA(cudaStreamSynchronize(h->stream));
}

}  // namespace

// the step's exchange between ranks (declared in cw_handle.cuh, called by the launcher of either form)
namespace cw {

CrossPlan cross_plan(const cw_handle* h, const std::vector<int>& pend) {
  CrossPlan c;
  std::vector<const RBox*> rb;
  for (int set : pend)
    for (const RBox& r : h->hs[set].r) {
      bool dup = false;
      for (const RBox* y : rb)
        dup |= y->me == r.me && y->t == r.t && y->fid == r.fid && y->send.i0 == r.send.i0 && y->send.j0 == r.send.j0;
      if (!dup) rb.push_back(&r);
    }
  std::stable_sort(rb.begin(), rb.end(), [](const RBox* a, const RBox* b) {
    return a->src_rank != b->src_rank ? a->src_rank < b->src_rank : a->dst_rank < b->dst_rank;
  });
  size_t so = 0, ro = 0;
  for (size_t g0 = 0; g0 < rb.size();) {
    size_t g1 = g0;
    while (g1 < rb.size() && rb[g1]->src_rank == rb[g0]->src_rank && rb[g1]->dst_rank == rb[g0]->dst_rank) ++g1;
    const size_t seg_s = so, seg_r = ro;
    for (size_t n = g0; n < g1; ++n) {
      const RBox& r = *rb[n];
      const long long wi = r.send.i1 - r.send.i0, wij = wi * (r.send.j1 - r.send.j0);
      if (r.has_send) {  // element (i, j, k) of the box at so + (i - i0) + (j - j0) wi + k wi wj of the send region
        XchgBox b = r.send;
        b.dst = nullptr;
        b.dst_ind = nullptr;
        b.dsj = int(wi);
        b.dsk = int(wij);
        b.doff = (long long)so - r.send.i0 - (long long)r.send.j0 * wi;
        c.pk.push_back(b);
        c.role.push_back(CrossPlan::Entry{0, r.dst_rank, &r, so});
        so += size_t(r.send.ncell);
      }
      if (r.has_recv) {
        XchgBox b = r.recv;
        b.src = nullptr;
        b.src_ind = nullptr;
        b.ssj = int(wi);
        b.ssk = int(wij);
        b.soff = (long long)ro - r.recv.i0 - (long long)r.recv.j0 * wi;
        c.unpk.push_back(b);
        c.role.push_back(CrossPlan::Entry{1, r.src_rank, &r, ro});
        ro += size_t(r.recv.ncell);
      }
    }
    const RBox& r0 = *rb[g0];
    if (h->loopback) c.copies.push_back(XCopy{seg_s, seg_r, so - seg_s});
    else if (r0.src_rank == h->rank) c.sends.push_back(Xfer{r0.dst_rank, seg_s, so - seg_s});
    else c.recvs.push_back(Xfer{r0.src_rank, seg_r, ro - seg_r});
    g0 = g1;
  }
  c.send_n = so;
  c.recv_n = ro;
  return c;
}

void nccl_exchange(cw_handle* h, const HaloTable& t, char* sbuf, char* rbuf, size_t esz) {
  const NcclApi& N = nccl_api();
  if (!N.ok || !h->comm) throw std::runtime_error("decomposition over ranks: no NCCL communicator");
  auto comm = static_cast<ncclComm_t>(h->comm);
  nccl_check(N, N.GroupStart(), "ncclGroupStart");
  ncclResult_t r = ncclSuccess;
  for (const Xfer& x : t.sends)
    if (r == ncclSuccess) r = N.Send(sbuf + x.off * esz, x.n * esz, ncclInt8, x.peer, comm, h->stream);
  for (const Xfer& x : t.recvs)
    if (r == ncclSuccess) r = N.Recv(rbuf + x.off * esz, x.n * esz, ncclInt8, x.peer, comm, h->stream);
  const ncclResult_t e = N.GroupEnd();
  nccl_check(N, r, "ncclSend / ncclRecv");
  nccl_check(N, e, "ncclGroupEnd");
}


}  // namespace cw

// cw_check_div_const: cw_div_const against __ddiv_rn for c = 60 and 12 on n operands each (the kinds of
// tests/div_const_check.c); counts[0] = checked, counts[1] = mismatches
__device__ __forceinline__ unsigned long long dc_mix(unsigned long long z) {  // splitmix64's output function
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__global__ void k_check_div_const(unsigned long long n, unsigned long long seed, unsigned long long* counts) {
  unsigned long long bad = 0, done = 0;
  const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (unsigned long long t = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; t < n; t += stride) {
    const unsigned long long u = dc_mix(seed + 0x9E3779B97F4A7C15ull * (2 * t + 1));
    const unsigned long long v = dc_mix(seed + 0x9E3779B97F4A7C15ull * (2 * t + 2));
    for (int ci = 0; ci < 2; ++ci) {
      const double c = ci == 0 ? 60.0 : 12.0, r = ci == 0 ? 1.0 / 60.0 : 1.0 / 12.0;
      double x;
      const int kind = int(t % 3);
      if (kind == 0) {
        x = __longlong_as_double((long long)u);
      } else if (kind == 1) {
        const unsigned long long e = 1023ull - 900ull + v % 1801ull;
        const double q = __longlong_as_double((long long)((u & 0x800FFFFFFFFFFFFFull) | (e << 52)));
        const double ulp = nextafter(fabs(q), __longlong_as_double(0x7FF0000000000000ll)) - fabs(q);
        x = __fma_rn(c, q, copysign(__dmul_rn(__dmul_rn(c, ulp), 0.5), q));
      } else {
        const long long m = (long long)(v % 2000001ull) - 1000000ll;
        x = (u & 1) ? double(m) : __dmul_rn(c, double(m));
        const int steps = int((u >> 1) % 5) - 2;
        for (int k = 0; k < (steps < 0 ? -steps : steps); ++k)
          x = nextafter(x, steps < 0 ? -__longlong_as_double(0x7FF0000000000000ll) : __longlong_as_double(0x7FF0000000000000ll));
      }
      const double a = cw_div_const(x, c, r), b = __ddiv_rn(x, c);
      ++done;
      if (__double_as_longlong(a) != __double_as_longlong(b) && !(isnan(a) && isnan(b))) ++bad;
    }
  }
  atomicAdd(counts, done);
  if (bad) atomicAdd(counts + 1, bad);
}

// ---- a decomposed domain's fields as whole-domain arrays (cw_decomp_upload / _download)
// the layout of a field of member M in a run with one patch (tile::whole_layout, src/core/tiles.hpp:98)
cw_layout whole_layout(const Member& M, int field) {
  if (field >= CW_Q_1) return layout_make(M.g, 'M', 3, false);
  return field_layout(M.g, M.o, field);
}
// a whole-domain array as member M's allocation: every point of its window (the others 0)
std::vector<double> to_patch(const cw_layout& Lp, const cw_layout& Lw, const double* whole) {
  std::vector<double> v(size_t(Lp.total), 0.0);
  if (Lw.uniform) {
    std::copy(whole, whole + std::min(Lp.total, Lw.total), v.begin());
    return v;
  }
  for (int k = 0; k < Lp.nz; ++k)
    for (int j = Lp.wj0; j < Lp.wj1; ++j)
      for (int i = Lp.wi0; i < Lp.wi1; ++i)
        v[size_t(Lp.offset + i + j * Lp.sj + k * Lp.sk)] = whole[Lw.offset + i + j * Lw.sj + k * Lw.sk];
  return v;
}
// member M's points into the whole-domain array: the points it owns, with the domain's halo beyond its edges
void from_patch(const Member& M, const cw_layout& Lp, const cw_layout& Lw, const double* part, double* whole) {
  if (Lw.uniform) {
    std::copy(part, part + std::min(Lp.total, Lw.total), whole);
    return;
  }
  const Box o = owned_box(M, Lp.stagger);
  const int i0 = M.patch.i0 == 0 ? Lp.wi0 : o.i0, i1 = M.patch.i1 == M.g.nx ? Lp.wi1 : o.i1;
  const int j0 = (two_d(M.g) || M.patch.j0 == 0) ? Lp.wj0 : o.j0;
  const int j1 = (two_d(M.g) || M.patch.j1 == M.g.ny) ? Lp.wj1 : o.j1;
  for (int k = 0; k < Lp.nz; ++k)
    for (int j = j0; j < j1; ++j)
      for (int i = i0; i < i1; ++i)
        whole[Lw.offset + i + j * Lw.sj + k * Lw.sk] = part[size_t(Lp.offset + i + j * Lp.sj + k * Lp.sk)];
}
// upload a whole-domain array to member mi (a patch: its window)
void upload_whole(cw_handle* h, int mi, int field, int n, const double* host, size_t count) {
  const Member& M = h->m.at(size_t(mi));
  const Loc l = locate(h, mi, field, n);
  if (!M.patched) {
    copy_in(h, l, host, count);
    return;
  }
  const cw_layout Lw = whole_layout(M, field);
  if (count != size_t(Lw.total)) throw std::runtime_error("count != the field's whole-domain layout total");
  const std::vector<double> v = to_patch(l.L, Lw, host);
  copy_in(h, l, v.data(), v.size());
}

// ------------------------------------------------------------------ C ABI
extern "C" {

int cw_create(const cw_grid* g, const cw_options* o, cw_handle** out) {
  return guarded(nullptr, [&] {
    if (!g || !o || !out) throw std::runtime_error("null argument");
    auto h = std::make_unique<cw_handle>();
    h->precision = o->precision;
    h->m.push_back(make_member(*g, *o));
    CW_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    setup(h.get());
    *out = h.release();
    return 0;
  });
}

int cw_batch_create(int n, const cw_grid* g, const cw_options* o, cw_handle** out) {
  return guarded(nullptr, [&] {
    if (n < 0 || n > kMaxMembers || (n > 0 && !g) || !o || !out) throw std::runtime_error("bad batch arguments");
    auto h = std::make_unique<cw_handle>();
    h->precision = o[0].precision;
    for (int m = 0; m < n; ++m) {
      if (o[m].precision != h->precision) throw std::runtime_error("batch members must share the precision");
      h->m.push_back(make_member(g[m], o[m]));
      if (h->m.back().n_sound != h->m[0].n_sound) throw std::runtime_error("batch members must share n_sound");
    }
    CW_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    setup(h.get());
    *out = h.release();
    return 0;
  });
}

int cw_decomp_patch(const cw_grid* g, int px, int py, int t, int* box) {
  return guarded(nullptr, [&] {
    if (!g || !box || t < 0 || t >= px * py) throw std::runtime_error("bad decomposition arguments");
    if (const char* why = decomp_unsupported(*g, px, py)) throw std::runtime_error(why);
    const Box b = patch_box(*g, px, py, t);
    box[0] = b.i0; box[1] = b.i1; box[2] = b.j0; box[3] = b.j1;
    return 0;
  });
}

int cw_decomp_create(const cw_grid* g, const cw_options* o, int px, int py, cw_handle** out) {
  return guarded(nullptr, [&] {
    if (!out) throw std::runtime_error("null argument");
    auto h = decomp_handle(g, o, px, py, 0, 1, false);
    CW_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    setup(h.get());
    *out = h.release();
    return 0;
  });
}

int cw_nccl_unique_id(unsigned char* id) {
  return guarded(nullptr, [&] {
    if (!id) throw std::runtime_error("null argument");
    const NcclApi& N = nccl_api();
    if (!N.ok) throw std::runtime_error(N.err);
    ncclUniqueId u;
    nccl_check(N, N.GetUniqueId(&u), "ncclGetUniqueId");
    static_assert(sizeof(u) == 128, "ncclUniqueId is 128 bytes");
    std::memcpy(id, &u, sizeof(u));
    return 0;
  });
}

int cw_decomp_create_ranked(const cw_grid* g, const cw_options* o, int px, int py, int rank, int nranks,
                            const unsigned char* nccl_id, cw_handle** out) {
  return guarded(nullptr, [&] {
    if (!out) throw std::runtime_error("null argument");
    auto h = decomp_handle(g, o, px, py, rank, nranks, nccl_id == nullptr);
    CW_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    if (nranks > 1 && !h->loopback) {  // every rank calls this with the same id: ncclCommInitRank waits for all
      const NcclApi& N = nccl_api();
      if (!N.ok) throw std::runtime_error(N.err);
      ncclUniqueId u;
      std::memcpy(&u, nccl_id, sizeof(u));
      ncclComm_t comm = nullptr;
      nccl_check(N, N.CommInitRank(&comm, nranks, u, rank), "ncclCommInitRank");
      h->comm = comm;
    }
    try {
      setup(h.get());
    } catch (...) {
      if (h->comm) nccl_api().CommDestroy(static_cast<ncclComm_t>(h->comm));
      throw;
    }
    *out = h.release();
    return 0;
  });
}

static_assert(int(CW_FILL_MU1) == int(cw_handle::H_MU1) && int(CW_FILL_PREP0) == int(cw_handle::H_PREP0) &&
                  int(CW_FILL_FIN) == int(cw_handle::H_FIN) && int(CW_FILL_Q2) == int(cw_handle::H_Q2) &&
                  int(CW_FILL_WS1) == int(cw_handle::H_WS1) && int(CW_FILL_XK) == int(cw_handle::H_XK) &&
                  int(CW_FILL_XK) + 1 == int(cw_handle::H_N),
              "the fill point indices of cw_decomp_plan are the handle's");
int cw_decomp_plan(const cw_grid* g, const cw_options* o, int px, int py, int rank, int nranks, int nsets,
                   const int* sets, long long* out, int cap, int* n) {
  return guarded(nullptr, [&] {
    if (!n || nsets < 1 || !sets || (cap > 0 && !out)) throw std::runtime_error("bad arguments");
    auto h = decomp_handle(g, o, px, py, rank, nranks, false);
    for (Member& M : h->m) plan_member(M);
    DevTables<double> T;  // no device tables: the items carry layouts only
    build_halosets_t<double>(h.get(), T, false);
    std::vector<int> pend;
    for (int k = 0; k < nsets; ++k) {
      if (sets[k] < 0 || sets[k] >= cw_handle::H_N) throw std::runtime_error("no such fill point");
      pend.push_back(sets[k]);
    }
    const CrossPlan c = cross_plan(h.get(), pend);
    *n = int(c.role.size());
    for (size_t k = 0; k < c.role.size() && int(k) < cap; ++k) {
      const CrossPlan::Entry& e = c.role[k];
      const RBox& r = *e.box;
      const long long v[11] = {e.role, e.peer, r.me, r.t, r.fid, r.send.i0, r.send.i1, r.send.j0, r.send.j1,
                               r.send.nk, (long long)e.off};
      std::copy(v, v + 11, out + 11 * k);
    }
    return 0;
  });
}

int cw_decomp_upload(cw_handle* h, int field, int n, const double* host, size_t count) {
  return guarded(h, [&] {
    if (!h || !host || h->decomp_px == 0) throw std::runtime_error("not a decomposed domain");
    for (int mi = 0; mi < int(h->m.size()); ++mi) upload_whole(h, mi, field, n, host, count);
    CW_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
  });
}

int cw_decomp_download(cw_handle* h, int field, int n, double* host, size_t count) {
  return guarded(h, [&] {
    if (!h || !host || h->decomp_px == 0) throw std::runtime_error("not a decomposed domain");
    const cw_layout Lw = whole_layout(h->m[0], field);
    if (count != size_t(Lw.total)) throw std::runtime_error("count != the field's whole-domain layout total");
    std::fill(host, host + count, 0.0);
    for (int mi = 0; mi < int(h->m.size()); ++mi) {
      const Loc l = locate(h, mi, field, n);
      std::vector<double> part(size_t(l.L.total));
      copy_out(h, l, part.data(), part.size());
      from_patch(h->m[size_t(mi)], l.L, Lw, part.data(), host);
    }
    return 0;
  });
}

int cw_decomp_upload_case(cw_handle* h, cw_case* c) {
  if (!h || !c || h->decomp_px == 0) return -1;
  for (int mi = 0; mi < int(h->m.size()); ++mi) {
    const int rc = cw_member_upload_case(h, mi, c);
    if (rc) return rc;
  }
  return 0;
}

int cw_batch_add(cw_handle* h, const cw_grid* g, const cw_options* o, int* member) {
  return guarded(h, [&] {
    if (!h || !g || !o) throw std::runtime_error("null argument");
    if (h->decomp_px) throw std::runtime_error("a decomposed domain's patches are fixed");
    if (int(h->m.size()) >= kMaxMembers) throw std::runtime_error("the batch is full");
    if (o->precision != h->precision) throw std::runtime_error("batch members must share the precision");
    Member M = make_member(*g, *o);
    if (!h->m.empty() && M.n_sound != h->m[0].n_sound) throw std::runtime_error("batch members must share n_sound");
    CW_CUDA(cudaStreamSynchronize(h->stream));
    allocate_member(h, M);
    h->m.push_back(std::move(M));
    try {
      rebuild(h);
    } catch (...) {
      cudaFree(h->m.back().arena);
      h->m.pop_back();
      rebuild(h);
      throw;
    }
    if (member) *member = int(h->m.size()) - 1;
    return 0;
  });
}

int cw_batch_adopt(cw_handle* h, cw_handle* single, int* member) {
  return guarded(h, [&] {
    if (!h || !single || single == h) throw std::runtime_error("bad arguments");
    if (h->decomp_px || single->decomp_px) throw std::runtime_error("a decomposed domain's patches are fixed");
    if (single->m.size() != 1) throw std::runtime_error("the adopted handle must hold one domain");
    if (single->precision != h->precision) throw std::runtime_error("batch members must share the precision");
    if (int(h->m.size()) >= kMaxMembers) throw std::runtime_error("the batch is full");
    if (!h->m.empty() && single->m[0].n_sound != h->m[0].n_sound) throw std::runtime_error("batch members must share n_sound");
    CW_CUDA(cudaStreamSynchronize(single->stream));
    CW_CUDA(cudaStreamSynchronize(h->stream));
    invalidate_graph(single);
    free_tables(single);
    h->m.push_back(std::move(single->m[0]));  // the domain's allocation changes hands, its contents stay
    single->m.clear();
    rebuild(h);
    if (member) *member = int(h->m.size()) - 1;
    return 0;
  });
}

int cw_batch_release(cw_handle* h, int member, cw_handle** out) {
  return guarded(h, [&] {
    if (!h || !out || member < 0 || member >= int(h->m.size())) throw std::runtime_error("member index out of range");
    if (h->decomp_px) throw std::runtime_error("a decomposed domain's patches are fixed");
    CW_CUDA(cudaStreamSynchronize(h->stream));
    auto s = std::make_unique<cw_handle>();
    s->precision = h->precision;
    s->device = h->device;
    CW_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
    invalidate_graph(h);
    free_tables(h);
    s->m.push_back(std::move(h->m[size_t(member)]));  // the domain's allocation changes hands, its contents stay
    h->m.erase(h->m.begin() + member);
    build_tables(h);
    build_tables(s.get());
    *out = s.release();
    return 0;
  });
}

int cw_batch_remove(cw_handle* h, int member) {
  return guarded(h, [&] {
    if (!h || member < 0 || member >= int(h->m.size())) throw std::runtime_error("member index out of range");
    if (h->decomp_px) throw std::runtime_error("a decomposed domain's patches are fixed");
    CW_CUDA(cudaStreamSynchronize(h->stream));
    invalidate_graph(h);
    free_tables(h);
    cudaFree(h->m[size_t(member)].arena);
    h->m.erase(h->m.begin() + member);
    build_tables(h);
    return 0;
  });
}

int cw_footprint(const cw_grid* g, const cw_options* o, size_t* bytes) {
  return guarded(nullptr, [&] {
    if (!g || !o || !bytes) throw std::runtime_error("null argument");
    Member M = make_member(*g, *o);
    *bytes = plan_member(M).total;
    return 0;
  });
}

int cw_destroy(cw_handle* h) {
  if (!h) return 0;
  cudaStreamSynchronize(h->stream);
  invalidate_graph(h);  // the captured step holds the NCCL operations: released before the communicator
  free_tables(h);
  if (h->comm) nccl_api().CommDestroy(static_cast<ncclComm_t>(h->comm));
  cudaFree(h->staging);
  cudaFree(h->diag);
  cudaFree(h->diag_part);
  cudaFree(h->status_d);
  for (Member& M : h->m) cudaFree(M.arena);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  delete h;
  return 0;
}

int cw_members(cw_handle* h, int* out) {
  if (!h || !out) return -1;
  *out = int(h->m.size());
  return 0;
}

int cw_member_config(cw_handle* h, int mi, cw_grid* g, cw_options* o) {
  return guarded(h, [&] {
    if (!h || mi < 0 || mi >= int(h->m.size())) throw std::runtime_error("member index out of range");
    if (g) *g = h->m[size_t(mi)].g;
    if (o) *o = h->m[size_t(mi)].o;
    return 0;
  });
}

int cw_member_set_vertical(cw_handle* h, int mi, const cw_vertical* v) {
  return guarded(h, [&] {
    if (!h || !v) throw std::runtime_error("null argument");
    Member& M = h->m.at(size_t(mi));
    const int nz = M.g.nz, stride = nz + 2;
    std::vector<double> buf(24 * size_t(stride), 0.0);
    auto put = [&](int slot, const double* src, int cnt) {
      if (src) std::copy(src, src + cnt, buf.begin() + size_t(slot) * stride);
    };
    put(VA_ZNU, v->znu, nz); put(VA_ZNW, v->znw, nz + 1); put(VA_DNW, v->dnw, nz); put(VA_DN, v->dn, nz + 1);
    put(VA_RDNW, v->rdnw, nz); put(VA_RDN, v->rdn, nz + 1); put(VA_FNM, v->fnm, nz + 1); put(VA_FNP, v->fnp, nz + 1);
    put(VA_C1H, v->c1h, nz); put(VA_C2H, v->c2h, nz); put(VA_C1F, v->c1f, nz + 1); put(VA_C2F, v->c2f, nz + 1);
    put(VA_UB, v->u_base, nz); put(VA_VB, v->v_base, nz); put(VA_TB, v->t_base, nz); put(VA_ZB, v->z_base, nz);
    put(VA_C3H, v->c3h, nz); put(VA_C4H, v->c4h, nz); put(VA_C3F, v->c3f, nz + 1); put(VA_C4F, v->c4f, nz + 1);
    if (M.o.lbc) {  // LateralBC::set_dt (src/dyn/lateral_bc.cpp:198-211): width 5, spec_zone 1, relax_zone 4
      const int spec_zone = 1, relax_zone = 4;
      for (int loop = spec_zone + 1; loop <= spec_zone + relax_zone; ++loop) {
        const double num = double(spec_zone + relax_zone - loop), den = double(relax_zone - 1);
        buf[size_t(VA_FCX) * stride + loop - 1] = 0.1 / M.g.dt * num / den;
        buf[size_t(VA_GCX) * stride + loop - 1] = 1.0 / M.g.dt / 50.0 * num / den;
      }
    }
    CW_CUDA(cudaMemcpyAsync(M.vert, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CW_CUDA(cudaStreamSynchronize(h->stream));
    M.cf1 = v->cf1; M.cf2 = v->cf2; M.cf3 = v->cf3; M.cfn = v->cfn; M.cfn1 = v->cfn1; M.rdx = v->rdx; M.rdy = v->rdy;
    M.g.p_top = v->p_top;
    upload_tables(h);
    invalidate_graph(h);
    return 0;
  });
}
int cw_set_vertical(cw_handle* h, const cw_vertical* v) { return cw_member_set_vertical(h, 0, v); }

int cw_member_upload(cw_handle* h, int mi, int field, int n, const double* host, size_t count) {
  return guarded(h, [&] {
    if (!h || !host) throw std::runtime_error("null argument");
    copy_in(h, locate(h, mi, field, n), host, count);
    CW_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
  });
}
int cw_upload(cw_handle* h, int field, int n, const double* host, size_t count) {
  return cw_member_upload(h, 0, field, n, host, count);
}
int cw_member_download(cw_handle* h, int mi, int field, int n, double* host, size_t count) {
  return guarded(h, [&] {
    if (!h || !host) throw std::runtime_error("null argument");
    copy_out(h, locate(h, mi, field, n), host, count);
    return 0;
  });
}
int cw_download(cw_handle* h, int field, int n, double* host, size_t count) {
  return cw_member_download(h, 0, field, n, host, count);
}
// several fields, one synchronisation: FP64 fields copy directly; FP32 (mixed) fields go through one staging region
// per field (the staging buffer sized for all of them first, so that no reallocation happens between the copies)
int cw_upload_fields(cw_handle* h, int mi, int nf, const int* fields, const int* ns, const double* const* host,
                     const size_t* counts) {
  return guarded(h, [&] {
    upload_fields(h, mi, nf, fields, ns, host, counts, false);
    return 0;
  });
}
int cw_download_fields(cw_handle* h, int mi, int nf, const int* fields, const int* ns, double* const* host,
                       const size_t* counts) {
  return guarded(h, [&] {
    download_fields(h, mi, nf, fields, ns, host, counts, false);
    return 0;
  });
}
int cw_upload_windows(cw_handle* h, int mi, int nf, const int* fields, const int* ns, const double* const* host,
                      const size_t* counts) {
  return guarded(h, [&] {
    upload_fields(h, mi, nf, fields, ns, host, counts, true);
    return 0;
  });
}
int cw_download_windows(cw_handle* h, int mi, int nf, const int* fields, const int* ns, double* const* host,
                        const size_t* counts) {
  return guarded(h, [&] {
    download_fields(h, mi, nf, fields, ns, host, counts, true);
    return 0;
  });
}
int cw_member_field_layout(cw_handle* h, int mi, int field, int n, cw_layout* out) {
  return guarded(h, [&] {
    if (!h || !out) throw std::runtime_error("null argument");
    *out = locate(h, mi, field, n).L;
    return 0;
  });
}
int cw_field_layout(cw_handle* h, int field, int n, cw_layout* out) { return cw_member_field_layout(h, 0, field, n, out); }
int cw_field_device_ptr(cw_handle* h, int field, int n, void** out) {
  return guarded(h, [&] {
    if (!h || !out) throw std::runtime_error("null argument");
    const Loc l = locate(h, 0, field, n);
    *out = l.base + size_t(l.L.offset) * l.esz;
    return 0;
  });
}

int cw_member_set_lbc(cw_handle* h, int mi, int var, int side, const double* values, const double* tends, size_t count) {
  return guarded(h, [&] {
    if (!h || !values || !tends) throw std::runtime_error("null argument");
    Member& M = h->m.at(size_t(mi));
    if (!M.o.lbc) throw std::runtime_error("the handle has no lateral boundaries (lbc = 0)");
    if (var < 0 || var > 4 || side < 0 || side > 3) throw std::runtime_error("bad boundary variable or side");
    const size_t n = size_t(lbc_npos(M.g, var, side)) * lbc_nk(M.g, var) * kLbcWidth;
    if (count != n) throw std::runtime_error("LateralBC::set: wrong slab size");
    const Loc vl{M.slab[var] + M.slab_off[var][side] * M.esz, cw_layout{}, M.esz};
    const Loc tl{M.slab[var] + M.slab_off[var][4 + side] * M.esz, cw_layout{}, M.esz};
    for (const auto& [dst, src] : {std::pair{vl.base, values}, std::pair{tl.base, tends}}) {
      if (M.esz == 8) {
        CW_CUDA(cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyHostToDevice, h->stream));
      } else {
        std::vector<float> f(src, src + n);
        CW_CUDA(cudaMemcpyAsync(dst, f.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
      }
      CW_CUDA(cudaStreamSynchronize(h->stream));
    }
    return 0;
  });
}
int cw_set_lbc(cw_handle* h, int var, int side, const double* values, const double* tends, size_t count) {
  return cw_member_set_lbc(h, 0, var, side, values, tends, count);
}
int cw_member_set_lbc_scalar(cw_handle* h, int mi, int n, int side, const double* values, const double* tends, size_t count) {
  return guarded(h, [&] {
    if (!h || !values || !tends) throw std::runtime_error("null argument");
    Member& M = h->m.at(size_t(mi));
    if (!M.o.lbc) throw std::runtime_error("the handle has no lateral boundaries (lbc = 0)");
    if (n < 0 || n >= M.o.n_scalars || side < 0 || side > 3) throw std::runtime_error("bad scalar or side");
    const size_t cnt = size_t(side < 2 ? M.g.ny : M.g.nx) * M.g.nz * kLbcWidth;
    if (count != cnt) throw std::runtime_error("LateralBC::set_scalar: wrong slab size");
    for (int half = 0; half < 2; ++half) {
      char* dst = M.qslab[n] + M.qslab_off[n][half * 4 + side] * M.esz;
      const double* src = half ? tends : values;
      if (M.esz == 8) {
        CW_CUDA(cudaMemcpyAsync(dst, src, cnt * 8, cudaMemcpyHostToDevice, h->stream));
      } else {
        std::vector<float> f(src, src + cnt);
        CW_CUDA(cudaMemcpyAsync(dst, f.data(), cnt * 4, cudaMemcpyHostToDevice, h->stream));
      }
      CW_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (!M.q_have[n]) {
      M.q_have[n] = 1;
      upload_tables(h);
      invalidate_graph(h);
    }
    return 0;
  });
}
int cw_set_lbc_scalar(cw_handle* h, int n, int side, const double* values, const double* tends, size_t count) {
  return cw_member_set_lbc_scalar(h, 0, n, side, values, tends, count);
}
int cw_member_set_lbc_time(cw_handle* h, int mi, double dtbc) {
  return guarded(h, [&] {
    h->m.at(size_t(mi)).dtbc = dtbc;
    upload_tables(h);
    return 0;
  });
}
int cw_set_lbc_time(cw_handle* h, double dtbc) { return cw_member_set_lbc_time(h, 0, dtbc); }

int cw_step(cw_handle* h, int nsteps) {
  return guarded(h, [&] {
    if (!h || nsteps < 0) throw std::runtime_error("bad arguments");
    run_steps(h, nsteps);
    return 0;
  });
}
int cw_set_dt(cw_handle* h, double dt, int n_sound) {
  return guarded(h, [&] {
    if (n_sound < 2 || n_sound % 2) throw std::runtime_error("time_step_sound must be even and >= 2");
    for (Member& M : h->m) {
      M.g.dt = dt;
      M.n_sound = n_sound;
    }
    upload_tables(h);
    invalidate_graph(h);
    return 0;
  });
}
int cw_n_sound(cw_handle* h, int* out) {
  if (!h || !out) return -1;
  *out = h->m[0].n_sound;
  return 0;
}
int cw_set_stream(cw_handle* h, void* stream) {
  return guarded(h, [&] {
    CW_CUDA(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    if (stream) {
      h->stream = static_cast<cudaStream_t>(stream);
      h->own_stream = false;
    } else {
      CW_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
      h->own_stream = true;
    }
    return 0;
  });
}
// a barrier that nothing completes, waited on with the kernels' bounded wait (cw_selftest_wait)
static __global__ void k_selftest_wait(unsigned* status, long long cycles) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  const bool ok = cycles > 0 ? mbar_wait(&bar, 0, cycles) : mbar_wait(&bar, 0);
  if (!ok && threadIdx.x == 0) atomicOr(status, 1u);
}
// the device status word: a kernel that gave up a bounded wait, or refused an unaligned copy, left work undone
static void check_status(cw_handle* h) {
  if (!h->status_d) return;
  unsigned st = 0;
  CW_CUDA(cudaMemcpyAsync(&st, h->status_d, sizeof st, cudaMemcpyDeviceToHost, h->stream));
  CW_CUDA(cudaStreamSynchronize(h->stream));
  if (st == 0) return;
  CW_CUDA(cudaMemsetAsync(h->status_d, 0, sizeof st, h->stream));
  throw std::runtime_error((st & 1u) ? "a kernel's wait for its tensor copies timed out: the step is incomplete"
                                     : "a kernel refused an unaligned tensor copy: the step is incomplete");
}
int cw_sync(cw_handle* h) {
  return guarded(h, [&] {
    CW_CUDA(cudaStreamSynchronize(h->stream));
    CW_CUDA(cudaGetLastError());
    check_status(h);
    return 0;
  });
}
int cw_selftest_wait(cw_handle* h, long long cycles) {
  return guarded(h, [&] {
    if (!h || !h->status_d) throw std::runtime_error("no handle");
    k_selftest_wait<<<1, 32, 0, h->stream>>>(h->status_d, cycles);
    CW_CUDA(cudaGetLastError());
    return 0;
  });
}
const char* cw_last_error(cw_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }
int cw_launch_count(cw_handle* h, long long* out) {
  if (!h || !out) return -1;
  *out = h->launches_last;
  return 0;
}
// per-kernel device time of nsteps eager steps (CUDA events around every launch; the steps advance the state)
int cw_profile(cw_handle* h, int nsteps, int* nkernels) {
  return guarded(h, [&] {
    if (!h || !nkernels) throw std::runtime_error("null argument");
    const bool g = h->use_graph;
    h->use_graph = false;
    h->profiling = true;
    h->prof_ev.clear();
    try {
      run_steps(h, nsteps);
    } catch (...) {
      h->profiling = false;
      h->use_graph = g;
      throw;
    }
    h->profiling = false;
    h->use_graph = g;
    CW_CUDA(cudaStreamSynchronize(h->stream));
    h->prof_names.clear();
    h->prof_ms.clear();
    h->prof_n.clear();
    for (auto& [name, ev] : h->prof_ev) {
      float ms = 0;
      CW_CUDA(cudaEventElapsedTime(&ms, ev.first, ev.second));
      cudaEventDestroy(ev.first);
      cudaEventDestroy(ev.second);
      size_t k = 0;
      while (k < h->prof_names.size() && h->prof_names[k] != name) ++k;
      if (k == h->prof_names.size()) {
        h->prof_names.emplace_back(name);
        h->prof_ms.push_back(0);
        h->prof_n.push_back(0);
      }
      h->prof_ms[k] += ms;
      h->prof_n[k] += 1;
    }
    h->prof_ev.clear();
    *nkernels = int(h->prof_names.size());
    return 0;
  });
}
int cw_profile_entry(cw_handle* h, int idx, char* name, int len, double* ms, long long* launches) {
  if (!h || idx < 0 || idx >= int(h->prof_names.size())) return -1;
  if (name && len > 0) {
    std::strncpy(name, h->prof_names[idx].c_str(), size_t(len) - 1);
    name[len - 1] = 0;
  }
  if (ms) *ms = h->prof_ms[idx];
  if (launches) *launches = h->prof_n[idx];
  return 0;
}
int cw_check_div_const(unsigned long long n, unsigned long long seed, unsigned long long* checked,
                       unsigned long long* mismatches) {
  return guarded(nullptr, [&] {
    if (!checked || !mismatches) throw std::runtime_error("null argument");
    unsigned long long* d = nullptr;
    CW_CUDA(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
    cudaError_t e = cudaMemset(d, 0, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) {
      k_check_div_const<<<148 * 8, 256>>>(n, seed, d);
      e = cudaGetLastError();
    }
    unsigned long long hc[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(hc, d, sizeof hc, cudaMemcpyDeviceToHost);
    cudaFree(d);
    CW_CUDA(e);
    *checked = hc[0];
    *mismatches = hc[1];
    return 0;
  });
}

int cw_check_finite(cw_handle* h, int mi, int* field, int* n, int* i, int* j, int* k) {
  return guarded(h, [&] {
    if (!h || mi < 0 || mi >= int(h->m.size())) throw std::runtime_error("member index out of range");
    Member& M = h->m[size_t(mi)];
    if (!h->diag) CW_CUDA(cudaMalloc(&h->diag, sizeof(unsigned long long)));
    const unsigned long long none = ~0ull;
    CW_CUDA(cudaMemcpyAsync(h->diag, &none, sizeof(none), cudaMemcpyHostToDevice, h->stream));
    // the prognostic state, slot s: U_2 V_2 W_2 T_2 PH_2 MU_2 P AL, then Q_2 of each species
    const int ids[8] = {CW_U_2, CW_V_2, CW_W_2, CW_T_2, CW_PH_2, CW_MU_2, CW_P, CW_AL};
    const int nslot = 8 + M.o.n_scalars;
    const unsigned long long span = 1ull << 40;
    for (int sl = 0; sl < nslot; ++sl) {
      const Loc l = sl < 8 ? locate(h, mi, ids[sl], 0) : locate(h, mi, CW_Q_2, sl - 8);
      const cw_layout& L = l.L;
      const long long npts = (long long)L.nx * L.ny * L.nz;
      const unsigned blocks = unsigned((npts + 255) / 256);
      if (l.esz == 8)
        k_nonfinite<double><<<blocks, 256, 0, h->stream>>>(reinterpret_cast<const double*>(l.base) + L.offset, int(L.sj),
                                                            int(L.sk), L.nx, L.ny, L.nz, span * sl, h->diag);
      else
        k_nonfinite<float><<<blocks, 256, 0, h->stream>>>(reinterpret_cast<const float*>(l.base) + L.offset, int(L.sj),
                                                           int(L.sk), L.nx, L.ny, L.nz, span * sl, h->diag);
      CW_CUDA(cudaGetLastError());
    }
    unsigned long long key = none;
    CW_CUDA(cudaMemcpyAsync(&key, h->diag, sizeof(key), cudaMemcpyDeviceToHost, h->stream));
    CW_CUDA(cudaStreamSynchronize(h->stream));
    if (key == none) {
      if (field) *field = -1;
      return 0;
    }
    const int sl = int(key / span);
    const long long t = (long long)(key % span);
    const Loc l = sl < 8 ? locate(h, mi, ids[sl], 0) : locate(h, mi, CW_Q_2, sl - 8);
    if (field) *field = sl < 8 ? ids[sl] : CW_Q_2;
    if (n) *n = sl < 8 ? 0 : sl - 8;
    if (i) *i = int(t % l.L.nx);
    if (j) *j = int((t / l.L.nx) % l.L.ny);
    if (k) *k = int(t / ((long long)l.L.nx * l.L.ny));
    return 1;
  });
}

int cw_diagnostics(cw_handle* h, int mi, cw_diag* out) {
  return guarded(h, [&] {
    if (!h || !out || mi < 0 || mi >= int(h->m.size())) throw std::runtime_error("bad diagnostics arguments");
    if (h->precision == CW_FP64) diagnostics_t<double>(h, mi, h->t64, out);
    else diagnostics_t<float>(h, mi, h->t32, out);
    return 0;
  });
}

int cw_set_cfl_diagnostics(cw_handle* h, int on) {
  if (!h) return -1;
  h->cfl_on = on != 0;
  invalidate_graph(h);
  return 0;
}

int cw_cfl_max(cw_handle* h, int mi, double* vert, double* horiz) {
  return guarded(h, [&] {
    if (!h || !vert || !horiz || mi < 0 || mi >= int(h->m.size())) throw std::runtime_error("bad cfl arguments");
    if (!h->cfl_on) throw std::runtime_error("CFL diagnostics are off (cw_set_cfl_diagnostics)");
    unsigned long long b[6];
    CW_CUDA(cudaMemcpyAsync(b, h->cfl_d + 6 * size_t(mi), sizeof b, cudaMemcpyDeviceToHost, h->stream));
    CW_CUDA(cudaStreamSynchronize(h->stream));
    for (int r = 0; r < 3; ++r) {
      vert[r] = b[2 * r] ? __builtin_bit_cast(double, b[2 * r]) : 0.0;
      horiz[r] = b[2 * r + 1] ? __builtin_bit_cast(double, b[2 * r + 1]) : 0.0;
    }
    return 0;
  });
}

int cw_set_autotune(cw_handle* h, int on) {
  if (!h) return -1;
  h->autotune = on != 0;
  h->tuned = false;
  h->tune_steps_done = 0;
  h->tune_ms.clear();
  h->shape_choice.clear();
  h->q_march = false;
  invalidate_graph(h);
  return 0;
}
int cw_autotune_choice(cw_handle* h, const char* kernel, int* shape) {
  if (!h || !kernel || !shape) return -1;
  *shape = -1;
  if (!h->tuned) return 0;
  for (const auto& [n, sh] : h->shape_choice)
    if (n == kernel) *shape = sh;
  return 0;
}
int cw_use_device(int device) {
  return guarded(nullptr, [&] {
    CW_CUDA(cudaSetDevice(device));
    return 0;
  });
}

int cw_set_graph(cw_handle* h, int on) {
  if (!h) return -1;
  h->use_graph = on != 0;
  invalidate_graph(h);
  return 0;
}

// FieldT::fill_host for every field of a case, plus the vertical arrays and the boundary slabs
int cw_member_upload_case(cw_handle* h, int mi, cw_case* c) {
  if (!h || !c) return -1;
  cw_vertical v{};
  if (cw_case_vertical(c, &v) != 0) return -1;
  int rc = cw_member_set_vertical(h, mi, &v);
  if (rc) return rc;
  const Member& M = h->m.at(size_t(mi));
  // a patch of a decomposed domain takes its window of the case's whole-domain fields
  auto up = [&](int id, int n, const double* data, size_t count) {
    return guarded(h, [&] {
      upload_whole(h, mi, id, n, data, count);
      CW_CUDA(cudaStreamSynchronize(h->stream));
      return 0;
    });
  };
  for (int id = 0; id < CW_Q_1; ++id) {
    double* data = nullptr;
    cw_layout L{};
    cw_case_field(c, id, 0, &data, &L);
    rc = up(id, 0, data, size_t(L.total));
    if (rc) return rc;
  }
  for (int n = 0; n < M.o.n_scalars; ++n)
    for (int id : {CW_Q_1, CW_Q_2, CW_Q_TENDF}) {
      double* data = nullptr;
      cw_layout L{};
      cw_case_field(c, id, n, &data, &L);
      rc = up(id, n, data, size_t(L.total));
      if (rc) return rc;
    }
  if (M.o.lbc) {
    for (int var = 0; var < 5; ++var)
      for (int side = 0; side < 4; ++side) {
        double *vals = nullptr, *tends = nullptr;
        size_t cnt = 0;
        cw_case_lbc(c, 0, var, side, &vals, &tends, &cnt);
        rc = cw_member_set_lbc(h, mi, var, side, vals, tends, cnt);
        if (rc) return rc;
      }
    for (int n = 0; n < M.o.n_scalars; ++n)
      for (int side = 0; side < 4; ++side) {
        double *vals = nullptr, *tends = nullptr;
        size_t cnt = 0;
        if (cw_case_lbc(c, 1, n, side, &vals, &tends, &cnt) != 0) continue;
        rc = cw_member_set_lbc_scalar(h, mi, n, side, vals, tends, cnt);
        if (rc) return rc;
      }
    double dtbc = 0;
    cw_case_lbc_time(c, &dtbc);
    rc = cw_member_set_lbc_time(h, mi, dtbc);
  }
  return rc;
}
int cw_upload_case(cw_handle* h, cw_case* c) { return cw_member_upload_case(h, 0, c); }

}  // extern "C"

// ------------------------------------------------------------------ download without allocating
// cw_download stages an FP32 field through a host vector (it widens to double on the host). Some callers
// cannot allocate at that moment: a checkpoint or state dump written after an allocation has failed (host
// or device memory exhausted), or a serving loop that has committed the whole device-memory budget to
// resident domains. cw_download_noalloc widens on the device into a scratch array that is part of the
// library image (a file-scope __device__ array, no cudaMalloc), then copies it to the caller's buffer.
namespace {

constexpr size_t kNoallocScratchDoubles = CW_NOALLOC_SCRATCH_DOUBLES;  // 8 MiB
static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchDoubles];

// the scratch's address on each device, looked up once per device (the lookup may load the library's
// device code on that device: the set-up work of the first call)
constexpr int kNoallocMaxDevices = 64;
std::atomic<double*> g_noalloc_addr[kNoallocMaxDevices];
std::mutex g_noalloc_mu;

double* noalloc_scratch(int device) {
  double* p = g_noalloc_addr[device].load(std::memory_order_acquire);
  if (p) return p;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  p = g_noalloc_addr[device].load(std::memory_order_relaxed);
  if (p) return p;
  void* a = nullptr;
  if (cudaGetSymbolAddress(&a, g_noalloc_scratch) != cudaSuccess) return nullptr;
  p = static_cast<double*>(a);
  g_noalloc_addr[device].store(p, std::memory_order_release);
  return p;
}

}  // namespace

extern "C" int cw_download_noalloc(cw_handle* h, int field, int n, double* host, size_t count) {
  if (!h || !host || h->m.empty() || field < 0 || field >= CW_NFIELDS) return CW_NOALLOC_EBADARG;
  Member& M = h->m[0];
  const bool scalar = field >= CW_Q_1;
  if (scalar && (n < 0 || n >= M.o.n_scalars)) return CW_NOALLOC_EBADARG;
  const Loc l = locate(h, 0, field, scalar ? n : 0);  // arguments checked above: does not throw
  if (count != size_t(l.L.total)) return CW_NOALLOC_EBADARG;
  if (l.esz == 8) {  // FP64 storage: a plain copy, no scratch
    if (cudaMemcpyAsync(host, l.base, count * 8, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      return CW_NOALLOC_ECUDA;
    return 0;
  }
  if (count > kNoallocScratchDoubles) return CW_NOALLOC_ETOOBIG;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kNoallocMaxDevices) return CW_NOALLOC_ECUDA;
  if (device != h->device) return CW_NOALLOC_EBADARG;  // the scratch of another device than the handle's
  double* scratch = noalloc_scratch(device);
  if (!scratch) return CW_NOALLOC_ECUDA;
  const unsigned nel = unsigned(count);
  const unsigned blocks = std::min(4096u, (nel + 255u) / 256u);
  // an error left by an earlier asynchronous launch belongs to its caller: it is reported here but not
  // consumed (cudaPeekAtLastError); only the failure of this call's own launch is cleared
  if (cudaPeekAtLastError() != cudaSuccess) return CW_NOALLOC_ECUDA;
  k_widen<<<blocks, 256, 0, h->stream>>>(reinterpret_cast<const float*>(l.base), scratch, nel);
  if (cudaPeekAtLastError() != cudaSuccess) {
    (void)cudaGetLastError();
    return CW_NOALLOC_ECUDA;
  }
  if (cudaMemcpyAsync(host, scratch, count * 8, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return CW_NOALLOC_ECUDA;
  return 0;
}
