// SPDX-License-Identifier: GPL-3.0-or-later
// The handle of the dycore's host runtime: its members (domains), device tables, halo sets and step state,
// shared by the translation units that enqueue the step (cw_runtime.cu: the FP64 form; cw_step_mixed.cu: the
// mixed form).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <utility>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/cw_output.h"
#include "cw_fields.hpp"
#include "kernels_cb.cuh"
#include "kernels_diag.cuh"
#include "kernels_mp.cuh"

namespace cw {

#define CW_CUDA(x)                                                                          \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr size_t kAlign = 256;
inline size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }
// the base-state fields the mixed form also keeps in double (Member::b64)
constexpr int kB64Fields[3] = {CW_PB, CW_ALB, CW_PHB};
inline int b64_slot(int field) {
  for (int x = 0; x < 3; ++x)
    if (kB64Fields[x] == field) return x;
  return -1;
}

// the work fields of one domain beyond State / Tendencies / BaseState (SmallStep's fields)
enum Work { W_U_SAVE, W_V_SAVE, W_W_SAVE, W_T_SAVE, W_PH_SAVE, W_WW1, W_C2A, W_PM1, W_T_2SAVE, W_A, W_ALPHA, W_GAMMA,
            W_MU_SAVE, W_MUDF, W_MUAVE, W_W_RHS, W_T2A, W_XKMH, W_XKHH, W_N };
// W_XKMH, W_XKHH: per-point horizontal eddy viscosities (damp_opt 1 or km_opt 4 only; no storage otherwise)
inline bool xk_fields(const cw_options& o) { return o.damp_opt == 1 || o.km_opt == 4; }
inline bool work_used(int w, const cw_options& o) { return (w != W_XKMH && w != W_XKHH) || xk_fields(o); }
inline FieldKind work_kind(int w) {
  switch (w) {
    case W_U_SAVE: return {'U', 3, false};
    case W_V_SAVE: return {'V', 3, false};
    case W_W_SAVE: case W_PH_SAVE: case W_WW1: case W_A: case W_ALPHA: case W_GAMMA: case W_W_RHS: return {'W', 3, false};
    case W_MU_SAVE: case W_MUDF: case W_MUAVE: return {'M', 2, false};
    default: return {'M', 3, false};
  }
}

struct Member {
  cw_grid g{};
  cw_options o{};
  bool patched = false;  // a patch of a decomposed domain (cw_decomp_create): fields allocated for `patch` + halo
  Box patch{};
  int tid = -1;  // its patch number t = tx + px ty
  const Box* pbox() const { return patched ? &patch : nullptr; }
  int n_sound = 0;
  int esz = 8;  // element size of the fields (8: FP64 form, 4: mixed form)
  std::vector<cw_layout> L;         // CW_U_1 .. CW_COSA
  std::vector<char*> base;          // allocation of each field
  std::vector<cw_layout> LW;
  std::vector<char*> wbase;
  cw_layout Lq{};
  std::vector<char*> q1, qa, qb, qtf, qsc;  // scalar allocations; q_2 is qa or qb by the parity
  std::vector<char*> qpd;                    // PD face fluxes, 6 per species (dh, lo on x, y, z faces), when PD
  cw_layout Lpd[3]{};                        // their layouts: U, V, W staggering
  double* vert = nullptr;           // device 1-D arrays (double)
  size_t vert_off[24]{};
  char* slab[5] = {};               // LBC slabs per variable (values 4 sides, tendencies 4 sides)
  size_t slab_off[5][8]{};
  std::vector<char*> qslab;
  std::vector<std::array<size_t, 8>> qslab_off;
  std::vector<char> q_have;
  double dtbc = 0;
  int q_parity = 0;
  // the mixed form: double copies of PB, ALB, PHB (kB64Fields), written with every upload of those fields and read
  // by the double parts of the step (the equation of state, the hydrostatic integrations); nullptr in FP64
  char* b64[3] = {nullptr, nullptr, nullptr};
  char* arena = nullptr;  // the member's device allocation (every pointer above points into it)
  size_t arena_bytes = 0;
  double cf1 = 0, cf2 = 0, cf3 = 0, cfn = 0, cfn1 = 0, rdx = 0, rdy = 0;
};

// the members' kernel parameter packs and each pack's block count per index range
template <class R, int NM>
struct Packs {
  std::vector<Pack<R, NM>> p;
  std::vector<std::array<std::array<int, kNumShapes>, kNumKinds>> blocks;  // [pack][kind][shape]
};
template <class R>
struct DevTables {  // the kernels' views of the members and the device scalar tables
  Packs<R, 1> one;   // a single domain
  Packs<R, 0> many;  // a batch: one pack over every member, its descriptors in device memory
  V3<R>* qtab = nullptr;  // per member: q1, q2, qn, qtf, qscale, 6 PD faces (kQTab x n_scalars)
  Slabs<R>* lbcq = nullptr;
  Dom<R>* doms_d = nullptr;  // the batch's member descriptors
  QMap* qmap = nullptr;       // per member and species: the tensor maps of the TMA-staged scalar update
};

// a fill point's fields (or the union of consecutive fill points') as a device table: one launch per pass
// whatever the number of fields (the batch path); for a decomposed domain also the exchange boxes, copied first
// A box of a decomposed domain's exchange whose two patches are on different ranks: patch `me` (on dst_rank)
// receives the points of the rectangle that patch t (on src_rank) owns. send: t's field -> the packed send buffer
// (when t is this process's); recv: the packed receive buffer -> me's field (when me is this process's).
struct RBox {
  int me, t, fid, src_rank, dst_rank;
  bool has_send, has_recv;
  XchgBox send, recv;
};
struct Xfer {  // a fill point's transfer with one rank: n elements at element offset off of the send / receive region
  int peer;
  size_t off, n;
};
struct XCopy {  // loopback transport: a send segment copied into its receive segment
  size_t soff, roff, n;
};

struct HaloTable {
  HaloField* f = nullptr;
  unsigned* start = nullptr;
  int nf = 0;
  unsigned total = 0;
  int has_oddface = 0;
  XchgBox* x = nullptr;  // the exchange between this process's patches, then the unpacking of received boxes
  unsigned* xstart = nullptr;
  int nx = 0;
  unsigned xtotal = 0;
  XchgBox* pk = nullptr;  // the packing of the boxes other ranks receive
  unsigned* pkstart = nullptr;
  int npk = 0;
  unsigned pktotal = 0;
  std::vector<Xfer> sends, recvs;  // over NCCL, in this order inside one group
  std::vector<XCopy> copies;       // loopback
};

struct HaloSetHost {
  std::vector<HaloField> f;
  std::vector<RBox> r;     // a decomposed domain over ranks: the boxes crossing between ranks
  std::vector<XchgBox> x;  // a decomposed domain: the points of other patches each patch receives first
  std::vector<HaloChunk<kHaloSmall>> small;  // the fields in one small chunk (most single domains), or
  std::vector<HaloChunk<kHaloLarge>> large;  // in large chunks
};

}  // namespace cw

using namespace cw;

constexpr int kTuneRounds = 2;  // autotuning: steps per block shape (one per round)

struct cw_handle {
  int precision = CW_FP64;
  std::vector<Member> m;
  int decomp_px = 0, decomp_py = 0;  // a decomposed domain (cw_decomp_create): its members are the px x py patches
  // a decomposed domain over ranks (cw_decomp_create_ranked): patch t is rank t % nranks's; this process holds the
  // patches of `rank` (every patch in the loopback form, whose exchanges between ranks are device copies)
  int rank = 0, nranks = 1;
  bool loopback = false;
  std::vector<Member> remote;  // the other ranks' patches: layouts only, for the exchange plan
  void* comm = nullptr;        // the ranks' NCCL communicator
  char* xbuf = nullptr;        // packed exchange buffers: send region (xsend_cap elements), then receive region
  size_t xsend_cap = 0, xrecv_cap = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = -1;  // the CUDA device current at create (every allocation of the handle is on it)
  DevTables<double> t64;
  DevTables<float> t32;
  double* dtbc_d = nullptr;  // per member: time since the boundary data, advanced by the step on the device
  unsigned long long* cfl_d = nullptr;  // per member: 3 stages x (vertical, horizontal) CFL maxima of the last step
  unsigned* status_d = nullptr;  // bit 0: a kernel's bounded wait for its copies gave up; bit 1: an unaligned copy refused
  bool q_tma = false;            // every member has the tensor maps: the TMA-staged k_q_march can run
  bool q_march = false;          // the autotuner chose k_q_march over the point kernel k_q_update
  bool cfl_on = false;                  // cw_set_cfl_diagnostics
  unsigned long long* diag = nullptr;  // cw_check_finite's result
  double* diag_part = nullptr;         // cw_diagnostics' per-level partials
  size_t diag_part_n = 0;
  double* staging = nullptr;  // FP32 field transfers: doubles converted on the device
  size_t staging_n = 0;
  int nzmax = 0;
  size_t cb_level_bytes = 0;  // one shared level array of a column block: (nz + 2) x CX doubles
  // halo sets of the fill points
  enum { H_MU1, H_PREP0, H_PREP1, H_SS0, H_UV, H_AC, H_POST, H_FIN, H_Q1PD, H_SCPD, H_Q2, H_END_P, H_WS0, H_WS1, H_MP,
         H_MP_P, H_XK, H_N };
  HaloSetHost hs[H_N];
  std::map<std::vector<int>, HaloTable> halo_tabs;  // batch: device tables of the fill points met while enqueuing
  std::vector<CopyDesc> copies;
  CopyDesc* copies_d = nullptr;
  long long* copies_start_d = nullptr;
  long long copies_total = 0;
  std::vector<CopyDesc> zeros;  // mudf reset
  CopyDesc* zeros_d = nullptr;
  long long* zeros_start_d = nullptr;
  long long zeros_total = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool graph_ok = false;
  bool use_graph = true;
  long long launches_step = 0;   // launches of one step
  long long launches_last = 0;   // launches of the last cw_step call
  std::string err;
  std::vector<void*> extra;      // other device allocations
  // per-kernel timing of eager steps (cw_profile): events around each launch
  // block-shape autotuning of the point kernels: the first kNumShapes steps each run every tunable kernel
  // with one shape (eager, timed per launch); then each kernel keeps its fastest shape
  bool autotune = false, tuned = false;  // (kTuneRounds steps per shape)
  int tuning_shape = -1, tune_steps_done = 0;
  std::vector<std::pair<std::string, int>> shape_choice;
  std::vector<std::pair<std::string, std::array<double, kNumShapes>>> tune_ms;
  bool profiling = false;
  std::vector<std::pair<const char*, std::pair<cudaEvent_t, cudaEvent_t>>> prof_ev;
  std::vector<std::string> prof_names;
  std::vector<double> prof_ms;
  std::vector<long long> prof_n;
};

namespace cw {

// a fill point's fields in launch chunks of NF descriptors
template <int NF>
void chunk_fields(const std::vector<HaloField>& f, std::vector<HaloChunk<NF>>& out) {
  for (size_t f0 = 0; f0 < f.size(); f0 += NF) {
    HaloChunk<NF> c{};
    c.nf = int(std::min(f.size() - f0, size_t(NF)));
    long long total = 0;
    for (int n = 0; n < c.nf; ++n) {
      c.f[n] = f[f0 + size_t(n)];
      c.start[n] = unsigned(total);
      total += c.f[n].ncell;
      c.has_oddface |= c.f[n].oddface_x;
    }
    if (total >= (1ll << 31)) throw std::runtime_error("a halo fill of more than 2^31 cells");
    c.start[c.nf] = unsigned(total);
    out.push_back(c);
  }
}

// the mixed form's step (cw_step_mixed.cu): enqueues one step of h on its stream (plan: no launch, only the
// tables the launches need), returns the launches
long long enqueue_mixed(cw_handle* h, bool plan);

// A decomposed domain over ranks: the boxes between ranks of a fill point (the union of the sets `pend`), each once,
// grouped by (sending rank, receiving rank) in ascending order and in list order inside a group -- the order both
// ranks of a pair derive -- packed into consecutive segments of the send region and unpacked from the same segments of
// the receive region. pk: the boxes this process packs (destination: the send region, doff the element offset),
// unpk: those it unpacks (source: the receive region, soff); the transfers per rank (or loopback copies); `role`
// lists every box as (0: packed, 1: unpacked) with its peer rank and region offset, in that order.
struct CrossPlan {
  std::vector<XchgBox> pk, unpk;
  std::vector<Xfer> sends, recvs;
  std::vector<XCopy> copies;
  struct Entry {
    int role, peer;
    const RBox* box;
    size_t off;
  };
  std::vector<Entry> role;
  size_t send_n = 0, recv_n = 0;
};
CrossPlan cross_plan(const cw_handle* h, const std::vector<int>& pend);

// a fill point's transfers between ranks (a decomposed domain over ranks): the send segments to their ranks and the
// receive segments from theirs, NCCL point-to-point in one group on the handle's stream (cw_runtime.cu)
void nccl_exchange(cw_handle* h, const HaloTable& t, char* sbuf, char* rbuf, size_t esz);

}  // namespace cw
