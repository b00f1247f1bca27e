// SPDX-License-Identifier: GPL-3.0-or-later
// Field catalogue and storage layout of the dycore's State / Tendencies / BaseState (host side).
// The layout is CPPWRF's (src/core/halo.cpp:12-48, Layout::make) so that a caller holding the reference's
// fields can hand their memory over unchanged: SoA, i fastest, k slowest, halo 3 in x (and in y when
// ny > 1), row pitch rounded up to 32 elements, element (0,0,0) at offset 8 + hy*pitch.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/cw_dycore.h"

namespace cw {

inline bool two_d(const cw_grid& g) { return g.ny == 1; }
inline int hy_of(const cw_grid& g) { return two_d(g) ? 0 : 3; }
inline int nxs(const cw_grid& g, char s) { return s == 'U' ? g.nx + 1 : g.nx; }
inline int nys(const cw_grid& g, char s) { return (s == 'V' && !two_d(g)) ? g.ny + 1 : g.ny; }
inline int nzs(const cw_grid& g, char s) { return s == 'W' ? g.nz + 1 : g.nz; }
inline bool flat_x(const cw_grid& g) { return g.bc_x == CW_BC_SPECIFIED || g.bc_x == CW_BC_OPEN; }
inline bool flat_y(const cw_grid& g) { return g.bc_y == CW_BC_SPECIFIED || g.bc_y == CW_BC_OPEN; }
inline bool specified(const cw_grid& g) { return g.bc_x == CW_BC_SPECIFIED || g.bc_y == CW_BC_SPECIFIED; }

// A patch of a decomposed domain: the mass points i0 <= i < i1, j0 <= j < j1 it owns (the domain's indices).
struct Box {
  int i0, i1, j0, j1;
};
// Layout::make for the whole domain, or (patch) for a patch and a halo of 3 around it, indexed with the domain's
// indices (the window [wi0, wi1) x [wj0, wj1); the east / north edge patches also hold the faces nx / ny and the
// lateral halos); uniform = horizontally uniform base field (1-D storage).
inline cw_layout layout_make(const cw_grid& g, char s, int rank, bool uniform, const Box* patch = nullptr) {
  cw_layout L{};
  L.nx = nxs(g, s);
  L.ny = nys(g, s);
  L.nz = rank == 3 ? nzs(g, s) : 1;
  L.rank = rank;
  L.uniform = uniform ? 1 : 0;
  L.stagger = s;
  if (uniform) {
    L.si = 0;
    L.sj = 0;
    L.sk = rank == 3 ? 1 : 0;
    L.offset = 0;
    L.total = L.nz;
    return L;
  }
  const int hy = hy_of(g);
  L.wi0 = -3;
  L.wi1 = L.nx + 3;
  L.wj0 = -hy;
  L.wj1 = L.ny + hy;
  if (patch) {
    L.wi0 = patch->i0 - 3;
    L.wi1 = (patch->i1 == g.nx ? L.nx : patch->i1) + 3;
    if (!two_d(g)) {
      L.wj0 = patch->j0 - 3;
      L.wj1 = (patch->j1 == g.ny ? L.ny : patch->j1) + 3;
    }
  }
  const int64_t pitch = (8 + (L.wi1 - L.wi0 - 3) + 31) / 32 * 32;
  L.si = 1;
  L.sj = two_d(g) ? 0 : pitch;
  const int64_t plane = pitch * (L.wj1 - L.wj0);
  L.sk = rank == 3 ? plane : 0;
  L.offset = 8 - (L.wi0 + 3) - int64_t(L.wj0) * L.sj;
  L.total = plane * (rank == 3 ? L.nz : 1);
  if (L.total >= (int64_t(1) << 31)) throw std::runtime_error("field too large for 32-bit view indexing");
  return L;
}

struct FieldKind {
  char stagger;
  int rank;
  bool uniform;
};

// stagger / rank / uniform of each field (src/dyn/state.cpp:10-24 State, Tendencies; :67-84 BaseState)
inline FieldKind field_kind(const cw_options& o, int id) {
  switch (id) {
    case CW_U_1: case CW_U_2: case CW_RU: case CW_RU_M: case CW_CQU: case CW_RU_TEND: case CW_RU_TENDF:
      return {'U', 3, false};
    case CW_V_1: case CW_V_2: case CW_RV: case CW_RV_M: case CW_CQV: case CW_RV_TEND: case CW_RV_TENDF:
      return {'V', 3, false};
    case CW_W_1: case CW_W_2: case CW_PH_1: case CW_PH_2: case CW_WW: case CW_RW: case CW_WW_M: case CW_CQW:
    case CW_RW_TEND: case CW_PH_TEND: case CW_RW_TENDF: case CW_PH_TENDF:
      return {'W', 3, false};
    case CW_MU_1: case CW_MU_2: case CW_MUT: case CW_MUTS: case CW_MU_TEND: case CW_RAINNC: case CW_RAINNCV:
      return {'M', 2, false};
    case CW_MUU: case CW_MUUS: return {'U', 2, false};
    case CW_MUV: case CW_MUVS: return {'V', 2, false};
    case CW_MUB: case CW_HT: return {'M', 2, o.flat != 0};
    case CW_PB: case CW_ALB: case CW_T_INIT: case CW_QV_BASE: return {'M', 3, o.flat != 0};
    case CW_PHB: return {'W', 3, o.flat != 0};
    case CW_MSFTX: case CW_MSFTY: case CW_F: case CW_E: case CW_SINA: case CW_COSA: return {'M', 2, o.mapped == 0};
    case CW_MSFUX: case CW_MSFUY: return {'U', 2, o.mapped == 0};
    case CW_MSFVX: case CW_MSFVY: case CW_MSFVX_INV: return {'V', 2, o.mapped == 0};
    default: return {'M', 3, false};  // t, p, al, alt, php, h_diabatic, t_tend(f), q
  }
}

inline cw_layout field_layout(const cw_grid& g, const cw_options& o, int id, const Box* patch = nullptr) {
  const FieldKind k = field_kind(o, id);
  return layout_make(g, k.stagger, k.rank, k.uniform, patch);
}

// Patch t = tx + px ty of a px x py decomposition (tile::set_domain, src/core/tiles.hpp:70-74): the mass points
// [tx nx / px, (tx + 1) nx / px) x [ty ny / py, (ty + 1) ny / py)
inline Box patch_box(const cw_grid& g, int px, int py, int t) {
  const int tx = t % px, ty = t / px;
  return Box{int(int64_t(tx) * g.nx / px), int(int64_t(tx + 1) * g.nx / px), int(int64_t(ty) * g.ny / py),
             int(int64_t(ty + 1) * g.ny / py)};
}
// why a px x py decomposition of g is refused (0: accepted)
inline const char* decomp_unsupported(const cw_grid& g, int px, int py) {
  if (px < 1 || py < 1 || px * py > 256) return "decomposition: 1 <= px, py and px * py <= 256";
  if (two_d(g) && py != 1) return "decomposition: a 2-D (x-z) domain is split along x only";
  if (g.bc_x == CW_BC_PERIODIC && px > 1) return "decomposition: a periodic direction is not split";
  if (g.bc_y == CW_BC_PERIODIC && py > 1) return "decomposition: a periodic direction is not split";
  if (g.nx / px < 6 || (!two_d(g) && g.ny / py < 6)) return "decomposition: patches of at least 6 x 6 points";
  return nullptr;
}

// n_sound: RK3::auto_sound_steps (src/dyn/rk3.cpp:69-72) when time_step_sound == 0
inline int sound_steps(const cw_grid& g, const cw_options& o) {
  if (o.time_step_sound > 0) return o.time_step_sound;
  const double spacing = g.dx < g.dy ? g.dx : g.dy;
  const int n = 2 * (int(300.0 * g.dt / spacing - 0.01) + 1);
  return n > 4 ? n : 4;
}

// LateralBC slab shapes (src/dyn/lateral_bc.cpp:222-238): npos per side, levels per variable
inline int lbc_npos(const cw_grid& g, int var, int side) {
  if (side == CW_XS || side == CW_XE) return var == CW_LBC_V ? g.ny + 1 : g.ny;
  return var == CW_LBC_U ? g.nx + 1 : g.nx;
}
inline int lbc_nk(const cw_grid& g, int var) {
  switch (var) {
    case CW_LBC_PH: return g.nz + 1;
    case CW_LBC_MU: return 1;
    default: return g.nz;
  }
}
constexpr int kLbcWidth = 5;

// The option set the dynamics step supports, with the reason of a refusal (0 = supported).
inline const char* unsupported(const cw_grid& g, const cw_options& o) {
  if (g.nx < 4 || g.ny < 1 || g.nz < 3) return "grid: need nx >= 4, ny >= 1, nz >= 3";
  if (!two_d(g) && g.ny < 4) return "grid: 3-D runs need ny >= 4";
  if ((g.bc_x == CW_BC_SPECIFIED) != (g.bc_y == CW_BC_SPECIFIED && !two_d(g)) && specified(g))
    return "specified boundaries: both directions of a 3-D grid";
  if (specified(g) && !o.lbc) return "specified boundaries need lbc = 1";
  if (o.lbc && !specified(g)) return "lbc = 1 needs specified boundaries";
  if (o.damp_opt < 0 || o.damp_opt > 3) return "damp_opt must be 0, 1, 2 or 3";
  if (o.damp_opt != 0 && !(o.zdamp > 0)) return "damp_opt 1, 2 and 3 need zdamp > 0";
  if (o.damp_opt == 2 && g.nz > 127) return "damp_opt 2: nz <= 127";
  if (o.hypsometric_opt != 1 && o.hypsometric_opt != 2) return "hypsometric_opt must be 1 or 2";
  if (o.diff_opt != 0 && !(o.diff_opt == 1 && (o.km_opt == 1 || o.km_opt == 4)))
    return "diffusion: diff_opt 0, or 1 with km_opt 1 or 4";
  if (o.h_adv_order != 5 && o.h_adv_order != 6) return "h_adv_order must be 5 or 6";
  if (o.v_adv_order != 3 && o.v_adv_order != 4) return "v_adv_order must be 3 or 4";
  if (o.n_moist < 0 || o.n_scalars < o.n_moist || o.n_scalars > 64) return "scalars: 0 <= n_moist <= n_scalars <= 64";
  if (g.nz > 126) return "nz must be <= 126 (the column limit of the reference's diffusion kernels)";
  if (o.precision != CW_FP64 && o.precision != CW_MIXED) return "precision must be CW_FP64 or CW_MIXED";
  const int ns = sound_steps(g, o);
  if (ns < 2 || ns % 2) return "time_step_sound must be even and >= 2";
  if (o.diff_6th_opt < 0 || o.diff_6th_opt > 2) return "diff_6th_opt must be 0, 1 or 2";
  if (o.mp_physics != 0 && o.mp_physics != 1) return "mp_physics must be 0 or 1 (Kessler)";
  if (o.mp_physics == 1 && o.n_moist < 3) return "Kessler microphysics needs the moist species qv, qc, qr (0, 1, 2)";
  if (o.mp_physics == 1 && !(o.mp_tend_lim > 0)) return "mp_tend_lim must be > 0";
  return nullptr;
}

}  // namespace cw
