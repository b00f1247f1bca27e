// SPDX-License-Identifier: GPL-3.0-or-later
// Run outputs in CPPWRF's formats (host side): the diag.csv line formatting of io::DiagWriter
// (src/io/output.cpp:344-389) and the snapshot writer io::SnapshotWriter (src/io/output.cpp:222-340) over the
// variables of dyn::snapshot_vars (src/dyn/diagnostics.cpp:82-153). The device reduction behind cw_diagnostics
// is in kernels_diag.cuh.
#include <unistd.h>

#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cw_output.h"
#include "cw_fields.hpp"

namespace {

thread_local std::string g_err;
std::atomic<unsigned long long> g_tmp_counter{0};

template <class F>
int guarded_out(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// shortest round-trip text of a double (std::to_chars without a format, as DiagWriter::row)
void put_shortest(std::string& s, double v) {
  char b[64];
  auto [ptr, ec] = std::to_chars(b, b + sizeof(b), v);
  s.append(b, size_t(ptr - b));
}
// JsonWriter::write_double: general format with max_digits10 significant digits
void put_json_double(std::string& s, double v) {
  if (std::isnan(v) || std::isinf(v)) throw std::runtime_error("snapshot: NaN or Infinity cannot be written to JSON");
  char b[64];
  auto [ptr, ec] = std::to_chars(b, b + sizeof(b), v, std::chars_format::general, std::numeric_limits<double>::max_digits10);
  s.append(b, size_t(ptr - b));
}
// JsonWriter::escape_string
std::string json_string(const std::string& t) {
  std::string r = "\"";
  for (unsigned char c : t) {
    switch (c) {
      case '"': r += "\\\""; break;
      case '\\': r += "\\\\"; break;
      case '\b': r += "\\b"; break;
      case '\f': r += "\\f"; break;
      case '\n': r += "\\n"; break;
      case '\r': r += "\\r"; break;
      case '\t': r += "\\t"; break;
      default:
        if (c < 0x20) {
          char hex[8];
          std::snprintf(hex, sizeof(hex), "\\u%04x", c);
          r += hex;
        } else {
          r.push_back(char(c));
        }
    }
  }
  return r + "\"";
}

int emit(const std::string& s, char* buf, size_t n) {
  if (!buf || n < s.size() + 1) return -1;
  std::memcpy(buf, s.data(), s.size());
  buf[s.size()] = 0;
  return int(s.size());
}

// a sibling temporary of target (make_temp_path of the reference: name.tmp.<pid>_<counter>)
std::filesystem::path temp_of(const std::filesystem::path& target) {
  return target.parent_path() / (target.filename().string() + ".tmp." + std::to_string(::getpid()) + "_" +
                                 std::to_string(++g_tmp_counter));
}

void write_atomic(const std::filesystem::path& target, const void* data, size_t bytes) {
  const std::filesystem::path tmp = temp_of(target);
  {
    std::ofstream out(tmp, std::ios::binary | std::ios::out | std::ios::trunc);
    if (!out.is_open()) throw std::runtime_error("snapshot: cannot open " + tmp.string());
    out.write(static_cast<const char*>(data), std::streamsize(bytes));
    out.close();
    if (!out) {
      std::error_code ec;
      std::filesystem::remove(tmp, ec);
      throw std::runtime_error("snapshot: cannot write " + tmp.string());
    }
  }
  std::error_code ec;
  std::filesystem::rename(tmp, target, ec);
  if (ec) {
    std::filesystem::remove(tmp, ec);
    throw std::runtime_error("snapshot: cannot rename " + tmp.string() + " to " + target.string());
  }
}

struct Var {
  std::string name;
  char stagger;
  int nx, ny, nz;
  std::vector<double> v;  // (k, j, i)
};

}  // namespace

extern "C" {

const char* cw_output_last_error(void) { return g_err.c_str(); }

int cw_diag_header(char* buf, size_t n) {
  return emit("step,time,max_abs_u,max_abs_v,max_abs_w,min_th_pert,max_th_pert,dry_mass,theta_mass,total_energy,wall_s",
              buf, n);
}

int cw_diag_format_row(long long step, double time, const cw_diag* d, double wall_s, char* buf, size_t n) {
  if (!d) return -1;
  // DomainRunner::do_diag (src/cases/domain_runner.cpp:1146-1152): the step number is written as a double
  const double vals[11] = {double(step), time, d->max_abs_u, d->max_abs_v, d->max_abs_w, d->min_th_pert, d->max_th_pert,
                           d->dry_mass, d->theta_mass, d->total_energy, wall_s};
  std::string s;
  for (int c = 0; c < 11; ++c) {
    if (c) s += ',';
    put_shortest(s, vals[c]);
  }
  return emit(s, buf, n);
}

int cw_snapshot_write_host(const char* dir, long long step, double time, const cw_grid* g, const cw_options* o,
                           const cw_snapshot_fields* f, const char* const* q_names) {
  return guarded_out([&] {
    if (!dir || !g || !o || !f) throw std::runtime_error("snapshot: null argument");
    if (!f->u_2 || !f->v_2 || !f->w_2 || !f->t_2 || !f->p || !f->ph_2 || !f->mu_2 || !f->pb || !f->phb || !f->t_init ||
        !f->mub || (o->n_scalars > 0 && !f->q_2) || (o->mp_physics != 0 && (!f->rainnc || !f->rainncv)))
      throw std::runtime_error("snapshot: a field array is missing");
    using namespace cw;
    auto lay = [&](int id) { return field_layout(*g, *o, id); };
    const cw_layout Lu = lay(CW_U_2), Lv = lay(CW_V_2), Lw = lay(CW_W_2), Lm = lay(CW_T_2), Lph = lay(CW_PH_2),
                    Lmu = lay(CW_MU_2), Lpb = lay(CW_PB), Lphb = lay(CW_PHB), Lti = lay(CW_T_INIT), Lmub = lay(CW_MUB),
                    Lq = lay(CW_Q_2);
    auto at = [](const double* a, const cw_layout& L, int i, int j, int k) {
      return a[L.offset + i * L.si + j * L.sj + k * L.sk];
    };
    constexpr double t0 = 300.0, gr = 9.81, rvovrd = 461.6 / 287.0;  // src/core/constants.hpp:5-15
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const bool moist = o->n_moist > 0;  // species 0 is qv (State::P_QV >= 0)
    std::vector<Var> vars;
    auto add = [&](const std::string& name, char st, int vx, int vy, int vz, const std::function<double(int, int, int)>& fn) {
      Var v{name, st, vx, vy, vz, std::vector<double>(size_t(vx) * vy * vz)};
      for (int k = 0; k < vz; ++k)
        for (int j = 0; j < vy; ++j)
          for (int i = 0; i < vx; ++i) v.v[(size_t(k) * vy + j) * vx + i] = fn(i, j, k);
      vars.push_back(std::move(v));
    };
    const int nyv = nys(*g, 'V');
    add("u", 'U', nx + 1, ny, nz, [&](int i, int j, int k) { return at(f->u_2, Lu, i, j, k); });
    add("v", 'V', nx, nyv, nz, [&](int i, int j, int k) { return at(f->v_2, Lv, i, j, k); });
    add("w", 'W', nx, ny, nz + 1, [&](int i, int j, int k) { return at(f->w_2, Lw, i, j, k); });
    auto theta = [&](int i, int j, int k) {  // dry theta (t_2 holds theta_m - t0 with moisture)
      const double tm = at(f->t_2, Lm, i, j, k) + t0;
      return !moist ? tm : tm / (1.0 + rvovrd * at(f->q_2[0], Lq, i, j, k));
    };
    add("th_pert", 'M', nx, ny, nz, [&](int i, int j, int k) { return theta(i, j, k) - t0 - at(f->t_init, Lti, i, j, k); });
    add("theta", 'M', nx, ny, nz, theta);
    if (moist) add("theta_m", 'M', nx, ny, nz, [&](int i, int j, int k) { return at(f->t_2, Lm, i, j, k) + t0; });
    add("p", 'M', nx, ny, nz, [&](int i, int j, int k) { return at(f->p, Lm, i, j, k) + at(f->pb, Lpb, i, j, k); });
    add("p_pert", 'M', nx, ny, nz, [&](int i, int j, int k) { return at(f->p, Lm, i, j, k); });
    add("ph", 'W', nx, ny, nz + 1, [&](int i, int j, int k) { return at(f->ph_2, Lph, i, j, k) + at(f->phb, Lphb, i, j, k); });
    add("mu", 'M', nx, ny, 1, [&](int i, int j, int) { return at(f->mu_2, Lmu, i, j, 0) + at(f->mub, Lmub, i, j, 0); });
    add("mu_pert", 'M', nx, ny, 1, [&](int i, int j, int) { return at(f->mu_2, Lmu, i, j, 0); });
    add("z_m", 'M', nx, ny, nz, [&](int i, int j, int k) {
      return 0.5 * (at(f->ph_2, Lph, i, j, k) + at(f->ph_2, Lph, i, j, k + 1) + at(f->phb, Lphb, i, j, k) +
                    at(f->phb, Lphb, i, j, k + 1)) / gr;
    });
    for (int n = 0; n < o->n_scalars; ++n) {
      if (!f->q_2[n]) throw std::runtime_error("snapshot: scalar array missing");
      static const char* const kessler[3] = {"qv", "qc", "qr"};
      std::string name = q_names && q_names[n] ? std::string(q_names[n])
                         : (moist && n == 0) || (o->mp_physics == 1 && n < 3) ? std::string(kessler[n])
                                                                              : "q" + std::to_string(n);
      const double* q = f->q_2[n];
      add(name, 'M', nx, ny, nz, [&](int i, int j, int k) { return at(q, Lq, i, j, k); });
    }
    if (o->mp_physics != 0) {  // PhysicsCoupling::rainnc, rainncv: the snapshot's extra 2-D fields
      const cw_layout Lr = lay(CW_RAINNC);
      add("rainnc", 'M', nx, ny, 1, [&](int i, int j, int) { return at(f->rainnc, Lr, i, j, 0); });
      add("rainncv", 'M', nx, ny, 1, [&](int i, int j, int) { return at(f->rainncv, Lr, i, j, 0); });
    }
    // the binary file: the variables one after the other, contiguous (k, j, i), little-endian float64
    size_t total = 0;
    for (const Var& v : vars) total += v.v.size();
    std::vector<double> bin;
    bin.reserve(total);
    for (const Var& v : vars) bin.insert(bin.end(), v.v.begin(), v.v.end());
    char base[32];
    std::snprintf(base, sizeof(base), "snap_%06lld", step);
    const std::filesystem::path d(dir);
    if (!d.empty()) std::filesystem::create_directories(d);
    write_atomic(d / (std::string(base) + ".bin"), bin.data(), bin.size() * sizeof(double));
    // the metadata, as JsonWriter writes it (no whitespace)
    std::string js = "{\"step\":" + std::to_string(step) + ",\"time\":";
    put_json_double(js, time);
    js += ",\"variables\":[";
    size_t off = 0;
    for (size_t a = 0; a < vars.size(); ++a) {
      const Var& v = vars[a];
      const size_t nb = v.v.size() * sizeof(double);
      if (a) js += ',';
      js += "{\"name\":" + json_string(v.name) + ",\"stagger\":" + json_string(std::string(1, v.stagger)) +
            ",\"shape\":[" + std::to_string(v.nz) + "," + std::to_string(v.ny) + "," + std::to_string(v.nx) +
            "],\"dtype\":\"float64\",\"offset\":" + std::to_string(off) + ",\"nbytes\":" + std::to_string(nb) + "}";
      off += nb;
    }
    js += "]}";
    write_atomic(d / (std::string(base) + ".json"), js.data(), js.size());
    return 0;
  });
}

int cw_snapshot_write(cw_handle* h, int member, const char* dir, long long step, double time,
                      const char* const* q_names) {
  return guarded_out([&] {
    if (!h) throw std::runtime_error("snapshot: null handle");
    cw_layout L{};
    auto get = [&](int id, int n, std::vector<double>& buf) {
      if (cw_member_field_layout(h, member, id, n, &L) != 0) throw std::runtime_error(cw_last_error(h));
      buf.resize(size_t(L.total));
      if (cw_member_download(h, member, id, n, buf.data(), buf.size()) != 0) throw std::runtime_error(cw_last_error(h));
      return buf.data();
    };
    cw_grid g{};
    cw_options o{};
    if (cw_member_config(h, member, &g, &o) != 0) throw std::runtime_error(cw_last_error(h));
    std::vector<double> u, v, w, t, p, ph, mu, pb, phb, ti, mub, rain, rainv;
    cw_snapshot_fields f{};
    f.u_2 = get(CW_U_2, 0, u); f.v_2 = get(CW_V_2, 0, v); f.w_2 = get(CW_W_2, 0, w); f.t_2 = get(CW_T_2, 0, t);
    f.p = get(CW_P, 0, p); f.ph_2 = get(CW_PH_2, 0, ph); f.mu_2 = get(CW_MU_2, 0, mu); f.pb = get(CW_PB, 0, pb);
    f.phb = get(CW_PHB, 0, phb); f.t_init = get(CW_T_INIT, 0, ti); f.mub = get(CW_MUB, 0, mub);
    std::vector<std::vector<double>> q(size_t(o.n_scalars));
    std::vector<const double*> qp(size_t(o.n_scalars));
    for (int n = 0; n < o.n_scalars; ++n) qp[size_t(n)] = get(CW_Q_2, n, q[size_t(n)]);
    f.q_2 = qp.data();
    if (o.mp_physics != 0) {
      f.rainnc = get(CW_RAINNC, 0, rain);
      f.rainncv = get(CW_RAINNCV, 0, rainv);
    }
    if (cw_snapshot_write_host(dir, step, time, &g, &o, &f, q_names) != 0) throw std::runtime_error(g_err);
    return 0;
  });
}

}  // extern "C"
