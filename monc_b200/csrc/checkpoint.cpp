// Checkpoint files in MONC's layout (checkpointer: writecheckpoint.F90:42-100 and its define_* /
// write_out_* routines, checkpointcommon.F90:11-81 for the names, readcheckpoint.F90 for what a
// restart reads), written as NetCDF classic with 64-bit offsets.  A serial MONC run writes the
// classic format (writecheckpoint.F90:53-58, NF90_CLOBBER) and nf90_open reads either, so these
// files restart MONC and MONC's serial checkpoints restart this library.
//
// The NetCDF classic format is written and parsed here directly: a big-endian header (magic
// "CDF\x02", record count, dimension, global attribute and variable lists, each variable with its
// dimension ids, attributes, type, size and 8-byte data offset) followed by each variable's data,
// padded to 4 bytes.  Variables are laid out as MONC defines them: the Fortran dimension order
// (z, y, x) is (x, y, zn) in the file, z varying fastest.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "mgpu_internal.h"

namespace mgpu {
namespace ncdf {

enum Type { NC_CHAR = 2, NC_INT = 4, NC_DOUBLE = 6 };
constexpr uint32_t TAG_DIM = 0x0A, TAG_VAR = 0x0B, TAG_ATT = 0x0C;

static int type_size(int t) { return t == NC_CHAR ? 1 : (t == NC_INT ? 4 : 8); }
static size_t pad4(size_t n) { return (n + 3) & ~(size_t)3; }

struct Att {
  std::string name, text;
};
struct Var {
  std::string name;
  int type = NC_DOUBLE;
  std::vector<int> dims;
  std::vector<Att> atts;
  std::vector<unsigned char> data;  // big-endian payload
  uint64_t begin = 0;
};

struct File {
  std::vector<std::pair<std::string, uint32_t>> dims;
  std::vector<Att> gatts;
  std::vector<Var> vars;

  int dim(const std::string& name) const {
    for (size_t q = 0; q < dims.size(); ++q)
      if (dims[q].first == name) return (int)q;
    return -1;
  }
  const Var* var(const std::string& name) const {
    for (const Var& v : vars)
      if (v.name == name) return &v;
    return nullptr;
  }
};

// ---- encoding -------------------------------------------------------------------------------
struct Out {
  std::vector<unsigned char> b;
  void u32(uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void u64(uint64_t v) {
    for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void name(const std::string& s) {
    u32((uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    while (b.size() % 4) b.push_back(0);
  }
};

static void put_be64(unsigned char* p, uint64_t v) {
  for (int q = 0; q < 8; ++q) p[q] = (unsigned char)(v >> (56 - 8 * q));
}
static void put_be32(unsigned char* p, uint32_t v) {
  for (int q = 0; q < 4; ++q) p[q] = (unsigned char)(v >> (24 - 8 * q));
}
static uint64_t get_be64(const unsigned char* p) {
  uint64_t v = 0;
  for (int q = 0; q < 8; ++q) v = (v << 8) | p[q];
  return v;
}
static uint32_t get_be32(const unsigned char* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

static void header(const File& f, Out& o) {
  o.b.clear();
  o.b.insert(o.b.end(), {'C', 'D', 'F', 2});
  o.u32(0);  // no record variables
  if (f.dims.empty()) { o.u32(0); o.u32(0); }
  else {
    o.u32(TAG_DIM);
    o.u32((uint32_t)f.dims.size());
    for (auto& d : f.dims) { o.name(d.first); o.u32(d.second); }
  }
  auto atts = [&](const std::vector<Att>& a) {
    if (a.empty()) { o.u32(0); o.u32(0); return; }
    o.u32(TAG_ATT);
    o.u32((uint32_t)a.size());
    for (const Att& t : a) {
      o.name(t.name);
      o.u32(NC_CHAR);
      o.u32((uint32_t)t.text.size());
      o.b.insert(o.b.end(), t.text.begin(), t.text.end());
      while (o.b.size() % 4) o.b.push_back(0);
    }
  };
  atts(f.gatts);
  if (f.vars.empty()) { o.u32(0); o.u32(0); return; }
  o.u32(TAG_VAR);
  o.u32((uint32_t)f.vars.size());
  for (const Var& v : f.vars) {
    o.name(v.name);
    o.u32((uint32_t)v.dims.size());
    for (int d : v.dims) o.u32((uint32_t)d);
    atts(v.atts);
    o.u32((uint32_t)v.type);
    const uint64_t vs = pad4(v.data.size());
    o.u32(vs > 0xFFFFFFFCull ? 0xFFFFFFFFu : (uint32_t)vs);
    o.u64(v.begin);
  }
}

static void write(File& f, const std::string& path) {
  Out o;
  header(f, o);  // sizes the header; the offsets follow from it
  uint64_t off = o.b.size();
  for (Var& v : f.vars) {
    v.begin = off;
    off += pad4(v.data.size());
  }
  header(f, o);
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) throw std::runtime_error("cannot open " + path + " for writing");
  bool ok = std::fwrite(o.b.data(), 1, o.b.size(), fp) == o.b.size();
  static const unsigned char zeros[4] = {0, 0, 0, 0};
  for (const Var& v : f.vars) {
    ok = ok && std::fwrite(v.data.data(), 1, v.data.size(), fp) == v.data.size();
    const size_t pad = pad4(v.data.size()) - v.data.size();
    ok = ok && std::fwrite(zeros, 1, pad, fp) == pad;
  }
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) throw std::runtime_error("short write to " + path);
}

// ---- decoding -------------------------------------------------------------------------------
struct In {
  const std::vector<unsigned char>& b;
  size_t p = 0;
  bool v2 = false;
  void need(size_t n) {
    if (p + n > b.size()) throw std::runtime_error("truncated NetCDF header");
  }
  uint32_t u32() { need(4); uint32_t v = get_be32(&b[p]); p += 4; return v; }
  uint64_t off() {
    if (v2) { need(8); uint64_t v = get_be64(&b[p]); p += 8; return v; }
    return u32();
  }
  std::string name() {
    uint32_t n = u32();
    need(pad4(n));
    std::string s((const char*)&b[p], n);
    p += pad4(n);
    return s;
  }
};

static std::vector<Att> read_atts(In& in) {
  std::vector<Att> a;
  uint32_t tag = in.u32(), n = in.u32();
  if (tag == 0) return a;
  if (tag != TAG_ATT) throw std::runtime_error("bad attribute list");
  for (uint32_t q = 0; q < n; ++q) {
    Att t;
    t.name = in.name();
    uint32_t type = in.u32(), cnt = in.u32();
    const size_t nb = (size_t)cnt * type_size((int)type);
    in.need(pad4(nb));
    if (type == NC_CHAR) t.text.assign((const char*)&in.b[in.p], cnt);
    in.p += pad4(nb);
    a.push_back(t);
  }
  return a;
}

static File read(const std::string& path) {
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) throw std::runtime_error("cannot open " + path);
  std::vector<unsigned char> b;
  unsigned char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, fp)) > 0) b.insert(b.end(), buf, buf + n);
  std::fclose(fp);
  if (b.size() < 8 || b[0] != 'C' || b[1] != 'D' || b[2] != 'F' || (b[3] != 1 && b[3] != 2))
    throw std::runtime_error(path + ": not a NetCDF classic file (HDF5-based NetCDF-4 files are not read)");
  In in{b};
  in.v2 = b[3] == 2;
  in.p = 4;
  File f;
  in.u32();  // records
  uint32_t tag = in.u32(), nd = in.u32();
  if (tag == TAG_DIM)
    for (uint32_t q = 0; q < nd; ++q) {
      std::string nm = in.name();
      f.dims.push_back({nm, in.u32()});
    }
  f.gatts = read_atts(in);
  tag = in.u32();
  uint32_t nv = in.u32();
  if (tag == TAG_VAR)
    for (uint32_t q = 0; q < nv; ++q) {
      Var v;
      v.name = in.name();
      uint32_t ndim = in.u32();
      for (uint32_t d = 0; d < ndim; ++d) v.dims.push_back((int)in.u32());
      v.atts = read_atts(in);
      v.type = (int)in.u32();
      in.u32();  // vsize
      v.begin = in.off();
      size_t cnt = 1;
      for (int d : v.dims) {
        if (d < 0 || d >= (int)f.dims.size()) throw std::runtime_error("bad dimension id");
        cnt *= f.dims[d].second;
      }
      const size_t nb = cnt * type_size(v.type);
      if (v.begin + nb > b.size()) throw std::runtime_error("variable " + v.name + " runs past the end of the file");
      v.data.assign(b.begin() + v.begin, b.begin() + v.begin + nb);
      f.vars.push_back(std::move(v));
    }
  return f;
}

// ---- typed payloads ---------------------------------------------------------------------------
static std::vector<unsigned char> doubles(const double* a, size_t n) {
  std::vector<unsigned char> d(8 * n);
  for (size_t q = 0; q < n; ++q) {
    uint64_t u;
    std::memcpy(&u, &a[q], 8);
    put_be64(&d[8 * q], u);
  }
  return d;
}
static std::vector<unsigned char> ints(const int32_t* a, size_t n) {
  std::vector<unsigned char> d(4 * n);
  for (size_t q = 0; q < n; ++q) put_be32(&d[4 * q], (uint32_t)a[q]);
  return d;
}
static double get_double(const Var& v, size_t q) {
  uint64_t u = get_be64(&v.data[8 * q]);
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}

}  // namespace ncdf

// ---- MONC's checkpoint layout -----------------------------------------------------------------
namespace {

constexpr int STRING_LENGTH = 150;  // datadefn.F90:10

std::string fmt(double x) {
  char s[40];
  std::snprintf(s, sizeof s, "%.17g", x);
  return s;
}
std::string fmt_bool(int b) { return b ? ".true." : ".false."; }

// the options this library's configuration carries, under MONC's option names
std::vector<std::pair<std::string, std::string>> options_of(const mgpu_config& c) {
  std::vector<std::pair<std::string, std::string>> o = {
      {"x_size", std::to_string(c.nx)}, {"y_size", std::to_string(c.ny)}, {"z_size", std::to_string(c.nz)},
      {"dxx", fmt(c.dxx)}, {"dyy", fmt(c.dyy)}, {"zztop", fmt(c.zztop)}, {"thref0", fmt(c.thref0)},
      {"rhobous", fmt(c.rhobous)}, {"surface_pressure", fmt(c.surface_pressure)},
      {"surface_reference_pressure", fmt(c.surface_reference_pressure)}, {"dtm", fmt(c.dtm)},
      {"passive_th", fmt_bool(c.passive_th)}, {"passive_q", fmt_bool(c.passive_q)},
      {"number_q_fields", std::to_string(c.number_q_fields)},
      {"use_viscosity_and_diffusion", fmt_bool(c.use_viscosity_and_diffusion)},
      {"use_surface_boundary_conditions", fmt_bool(c.use_surface_boundary_conditions)},
      {"type_of_surface_boundary_conditions", std::to_string(c.type_of_surface_boundary_conditions)},
      {"surface_sensible_heat_flux", fmt(c.surface_sensible_heat_flux)},
      {"surface_latent_heat_flux", fmt(c.surface_latent_heat_flux)},
      {"coriolis_enabled", fmt_bool(c.coriolis_enabled)}, {"fcoriol", fmt(c.fcoriol)},
      {"surface_geostrophic_wind_x", fmt(c.surface_geostrophic_wind_x)},
      {"surface_geostrophic_wind_y", fmt(c.surface_geostrophic_wind_y)},
      {"smag-subb", fmt(c.smag_subb)}, {"smag-subc", fmt(c.smag_subc)},
      {"simplecloud_enabled", fmt_bool(c.simplecloud_enabled)}, {"max_height_cloud", fmt(c.max_height_cloud)},
      {"fftsolver_enabled", fmt_bool(c.solver == MGPU_SOLVER_FFT)},
      {"iterativesolver_enabled", fmt_bool(c.solver == MGPU_SOLVER_ITERATIVE)},
      {"tolerance", fmt(c.tolerance)}, {"max_iterations", std::to_string(c.max_iterations)},
      {"cfltest_enabled", fmt_bool(c.cfl_enabled)}, {"cfl_frequency", std::to_string(c.cfl_frequency)},
      {"cfl_tollerance", fmt(c.cfl_tollerance)}, {"cfl_cvismax", fmt(c.cfl_cvismax)},
      {"cfl_cvelmax", fmt(c.cfl_cvelmax)}, {"cfl_dtmmax", fmt(c.cfl_dtmmax)}, {"cfl_dtmmin", fmt(c.cfl_dtmmin)},
      {"cfl_rincmax", fmt(c.cfl_rincmax)}, {"l_constant_dtm", fmt_bool(c.l_constant_dtm)},
      {"advection_flow_fields", c.advection_flow_fields == MGPU_ADVECT_TVD ? "tvd" : "pw"},
      {"advection_theta_field", "tvd"}, {"advection_q_fields", "tvd"},
      {"damping_enabled", fmt_bool(c.damping_enabled)}, {"dmptim", fmt(c.dmptim)}, {"zdmp", fmt(c.zdmp)},
      {"hdmp", fmt(c.hdmp)}, {"l_subs_pl_theta", fmt_bool(c.l_subs_pl_theta)},
      {"l_subs_pl_q", fmt_bool(c.l_subs_pl_q)}, {"subsidence_input_type", std::to_string(c.subsidence_input_type)},
      {"subsidence_local_theta", fmt_bool(c.subsidence_local_theta)},
      {"subsidence_local_q", fmt_bool(c.subsidence_local_q)},
      {"mean_profiles_enabled", fmt_bool(c.damping_enabled || c.l_subs_pl_theta || c.l_subs_pl_q)},
      {"galilean_transformation", fmt_bool(c.galilean_transformation)}, {"fix_ugal", fmt_bool(c.fix_ugal)},
      {"fix_vgal", fmt_bool(c.fix_vgal)}, {"ugal", fmt(c.ugal)}, {"vgal", fmt(c.vgal)}};
  if (c.rmlmax > 0.0) o.push_back({"rmlmax", fmt(c.rmlmax)});
  return o;
}

// key/value strings of a char variable (n, 2, STRING_LENGTH)
std::vector<unsigned char> kv_chars(const std::vector<std::pair<std::string, std::string>>& kv) {
  std::vector<unsigned char> d(kv.size() * 2 * STRING_LENGTH, 0);
  for (size_t q = 0; q < kv.size(); ++q) {
    std::memcpy(&d[(2 * q) * STRING_LENGTH], kv[q].first.data(), std::min<size_t>(kv[q].first.size(), STRING_LENGTH));
    std::memcpy(&d[(2 * q + 1) * STRING_LENGTH], kv[q].second.data(),
                std::min<size_t>(kv[q].second.size(), STRING_LENGTH));
  }
  return d;
}

std::string created_stamp() {
  std::time_t t = std::time(nullptr);
  std::tm tm{};
  localtime_r(&t, &tm);
  char s[64];
  // writecheckpoint.F90:112-115: day/month/year hour:minute:second
  std::snprintf(s, sizeof s, "%d/%d/%d %d:%d:%d", tm.tm_mday, tm.tm_mon + 1, tm.tm_year + 1900, tm.tm_hour, tm.tm_min,
                tm.tm_sec);
  return s;
}

const char* FIELD_NAMES[9] = {"u_nogal", "v_nogal", "w", "th", "zu", "zv", "zw", "zth", "p"};
// MONC's write order of the prognostic fields (writecheckpoint.F90:181-203 / define_prognostic_variables)
const int FIELD_ORDER[9] = {0, 4, 1, 5, 2, 6, 3, 7, 8};

// [nz][ny][nx] x-fastest <-> (x, y, z) z-fastest
void to_zfast(const double* a, int nx, int ny, int nz, double* out) {
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) out[((size_t)i * ny + j) * nz + k] = a[((size_t)k * ny + j) * nx + i];
}
void from_zfast(const double* a, int nx, int ny, int nz, double* out) {
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) out[((size_t)k * ny + j) * nx + i] = a[((size_t)i * ny + j) * nz + k];
}

}  // namespace

int checkpoint_write_host(const mgpu_config& c, const RefState& rs, const std::string& path,
                          const double* const* fields, const double* mean, const mgpu_checkpoint_meta& meta,
                          std::string& err) {
  using namespace ncdf;
  try {
    const int nx = c.nx, ny = c.ny, nz = c.nz, nq = c.number_q_fields;
    const size_t npt = (size_t)nx * ny * nz;
    File f;
    f.gatts = {{"title", "MONC checkpoint file"}, {"created", created_stamp()}};
    // dimensions in MONC's order (define_grid_dimensions, define_q_field_dimension,
    // define_options_variable, define_q_indices_variable)
    f.dims = {{"empty_dim", 1}, {"z", (uint32_t)nz}, {"zn", (uint32_t)nz}, {"y", (uint32_t)ny}, {"x", (uint32_t)nx}};
    if (nq > 0) f.dims.push_back({"q", (uint32_t)nq});
    const auto opts = options_of(c);
    f.dims.push_back({"string", (uint32_t)STRING_LENGTH});
    f.dims.push_back({"kvp", 2});
    f.dims.push_back({"number_options", (uint32_t)opts.size()});
    std::vector<std::pair<std::string, std::string>> qidx;
    if (nq > 0 && !c.passive_q) {
      qidx.push_back({"vapour", "1"});
      if (nq > 1) qidx.push_back({"cloud_liquid_mass", "2"});
      f.dims.push_back({"active_q_indicies", (uint32_t)qidx.size()});
    }
    const int dz = f.dim("z"), dzn = f.dim("zn"), dy = f.dim("y"), dx = f.dim("x"), dq = f.dim("q");
    auto var = [&](const std::string& name, int type, std::vector<int> dims, std::vector<unsigned char> data,
                   std::vector<Att> atts = {}) {
      Var v;
      v.name = name;
      v.type = type;
      v.dims = std::move(dims);
      v.data = std::move(data);
      v.atts = std::move(atts);
      f.vars.push_back(std::move(v));
    };
    var("options_database", NC_CHAR, {f.dim("number_options"), f.dim("kvp"), f.dim("string")}, kv_chars(opts));
    if (!qidx.empty())
      var("q_indicies", NC_CHAR, {f.dim("active_q_indicies"), f.dim("kvp"), f.dim("string")}, kv_chars(qidx));
    const std::vector<Att> metres = {{"units", "m"}};
    // grid (define_grid_variables, write_out_grid): top = n dx, bottom = 0 for a periodic domain
    var("x_resolution", NC_DOUBLE, {}, doubles(&c.dxx, 1), metres);
    const double xt = nx * c.dxx, yt = ny * c.dyy, zero = 0.0;
    var("x_top", NC_DOUBLE, {}, doubles(&xt, 1), metres);
    var("x_bottom", NC_DOUBLE, {}, doubles(&zero, 1), metres);
    var("y_resolution", NC_DOUBLE, {}, doubles(&c.dyy, 1), metres);
    var("y_top", NC_DOUBLE, {}, doubles(&yt, 1), metres);
    var("y_bottom", NC_DOUBLE, {}, doubles(&zero, 1), metres);
    var("z", NC_DOUBLE, {dz}, doubles(&rs.z[1], nz), metres);
    var("zn", NC_DOUBLE, {dzn}, doubles(&rs.zn[1], nz), metres);
    var("thref", NC_DOUBLE, {dz}, doubles(&rs.thref[1], nz));
    if (mean) {
      // mean: (3 + nq) rows of olz*bar, then (3 + nq) rows of olubar, olvbar, olthbar, olqbar(n);
      // writecheckpoint.F90:508-535 defines each one mean_profiles allocated
      const double* bar = mean + (size_t)(3 + nq) * nz;
      var("olubar", NC_DOUBLE, {dz}, doubles(bar, nz));
      var("olzubar", NC_DOUBLE, {dz}, doubles(mean, nz));
      var("olvbar", NC_DOUBLE, {dz}, doubles(bar + nz, nz));
      var("olzvbar", NC_DOUBLE, {dz}, doubles(mean + nz, nz));
      var("olthbar", NC_DOUBLE, {dz}, doubles(bar + 2 * nz, nz));
      var("olzthbar", NC_DOUBLE, {dz}, doubles(mean + 2 * nz, nz));
      if (nq > 0) {
        var("olqbar", NC_DOUBLE, {dq, dz}, doubles(bar + 3 * nz, (size_t)nq * nz));
        var("olzqbar", NC_DOUBLE, {dq, dz}, doubles(mean + 3 * nz, (size_t)nq * nz));
      }
    }
    std::vector<double> buf(npt);
    if (nq > 0) {
      for (int zq = 0; zq < 2; ++zq) {
        std::vector<double> all((size_t)nq * npt);
        for (int n = 0; n < nq; ++n) to_zfast(fields[9 + zq * nq + n], nx, ny, nz, &all[(size_t)n * npt]);
        var(zq ? "zq" : "q", NC_DOUBLE, {dq, dx, dy, dzn}, doubles(all.data(), all.size()));
      }
    }
    for (int q = 0; q < 9; ++q) {
      const int fi = FIELD_ORDER[q];
      to_zfast(fields[fi], nx, ny, nz, buf.data());
      var(FIELD_NAMES[fi], NC_DOUBLE, {dx, dy, dzn}, doubles(buf.data(), npt));
    }
    const int32_t zero_i = 0, one_i = 1;
    var("timestep", NC_INT, {}, ints(&meta.timestep, 1));
    var("time", NC_DOUBLE, {}, doubles(&meta.time, 1));
    var("ugal", NC_DOUBLE, {}, doubles(&meta.ugal, 1));
    var("vgal", NC_DOUBLE, {}, doubles(&meta.vgal, 1));
    const int32_t nq_i = nq;
    var("nqfields", NC_INT, {}, ints(&nq_i, 1));
    var("dtm", NC_DOUBLE, {}, doubles(&meta.dtm, 1));
    var("dtm_new", NC_DOUBLE, {}, doubles(&meta.dtm_new, 1));
    var("absolute_new_dtm", NC_DOUBLE, {}, doubles(&meta.absolute_new_dtm, 1));
    var("ntracers", NC_INT, {}, ints(&zero_i, 1));
    var("nradtracers", NC_INT, {}, ints(&zero_i, 1));
    var("normal_step", NC_INT, {}, ints(&one_i, 1));
    var("rad_last_time", NC_DOUBLE, {}, doubles(&zero, 1));
    var("last_cfl_timestep", NC_INT, {}, ints(&meta.last_cfl_timestep, 1));
    var("reconfig_timestep_offset", NC_INT, {}, ints(&zero_i, 1));
    write(f, path);
  } catch (std::exception& e) {
    err = e.what();
    return MGPU_ERR_ARGUMENT;
  }
  return MGPU_OK;
}

int checkpoint_read_host(const mgpu_config& c, const std::string& path, double* const* fields, double* mean,
                         int* has_mean, mgpu_checkpoint_meta& meta, std::string& err) {
  using namespace ncdf;
  try {
    const File f = read(path);
    const int nx = c.nx, ny = c.ny, nz = c.nz, nq = c.number_q_fields;
    const size_t npt = (size_t)nx * ny * nz;
    auto dim_is = [&](const char* d, int n) {
      int id = f.dim(d);
      if (id < 0 || (int)f.dims[id].second != n)
        throw std::runtime_error(std::string("dimension ") + d + " does not match the model (" + std::to_string(n) + ")");
    };
    dim_is("x", nx);
    dim_is("y", ny);
    dim_is("zn", nz);
    auto need = [&](const char* name) -> const Var& {
      const Var* v = f.var(name);
      if (!v) throw std::runtime_error(std::string("variable ") + name + " missing");
      return *v;
    };
    auto field = [&](const char* name, double* out, size_t slab) {
      const Var& v = need(name);
      if (v.type != NC_DOUBLE) throw std::runtime_error(std::string(name) + " is not double precision");
      if (v.data.size() < (slab + 1) * npt * 8) throw std::runtime_error(std::string(name) + " has the wrong size");
      std::vector<double> tmp(npt);
      for (size_t q = 0; q < npt; ++q) tmp[q] = get_double(v, slab * npt + q);
      from_zfast(tmp.data(), nx, ny, nz, out);
    };
    for (int q = 0; q < 9; ++q) field(FIELD_NAMES[q], fields[q], 0);
    if (nq > 0) {
      const Var* nv = f.var("nqfields");
      if (!nv || (int)get_be32(nv->data.data()) != nq) throw std::runtime_error("the file's nqfields differs from the model's");
      for (int n = 0; n < nq; ++n) {
        field("q", fields[9 + n], n);
        field("zq", fields[9 + nq + n], n);
      }
    }
    auto scalar_d = [&](const char* name, double dflt) {
      const Var* v = f.var(name);
      return v && v->type == NC_DOUBLE && v->data.size() >= 8 ? get_double(*v, 0) : dflt;
    };
    auto scalar_i = [&](const char* name, int dflt) {
      const Var* v = f.var(name);
      return v && v->type == NC_INT && v->data.size() >= 4 ? (int)get_be32(v->data.data()) : dflt;
    };
    meta.timestep = scalar_i("timestep", 0);
    meta.time = scalar_d("time", 0.0);
    meta.ugal = scalar_d("ugal", 0.0);
    meta.vgal = scalar_d("vgal", 0.0);
    meta.dtm = scalar_d("dtm", c.dtm);
    meta.dtm_new = scalar_d("dtm_new", meta.dtm);
    meta.absolute_new_dtm = scalar_d("absolute_new_dtm", meta.dtm);
    meta.last_cfl_timestep = scalar_i("last_cfl_timestep", 0);
    // readcheckpoint.F90:540-600 reads each mean profile that is present: here the olz*bar set
    // (has_mean 1) and, when it is complete too, the olubar, olvbar, olthbar, olqbar set (has_mean
    // 2; otherwise those rows are zero)
    *has_mean = 0;
    if (mean && f.var("olzubar") && f.var("olzvbar") && f.var("olzthbar") && (nq == 0 || f.var("olzqbar"))) {
      const size_t rows = (size_t)(3 + nq);
      auto read_set = [&](const char* const* names, const char* qname, double* out) {
        for (int r = 0; r < 3; ++r)
          for (int k = 0; k < nz; ++k) out[r * nz + k] = get_double(need(names[r]), k);
        for (int n = 0; n < nq; ++n)
          for (int k = 0; k < nz; ++k) out[(3 + n) * nz + k] = get_double(need(qname), (size_t)n * nz + k);
      };
      const char* zn[3] = {"olzubar", "olzvbar", "olzthbar"};
      read_set(zn, "olzqbar", mean);
      *has_mean = 1;
      double* bar = mean + rows * nz;
      std::fill(bar, bar + rows * nz, 0.0);
      if (f.var("olubar") && f.var("olvbar") && f.var("olthbar") && (nq == 0 || f.var("olqbar"))) {
        const char* bn[3] = {"olubar", "olvbar", "olthbar"};
        read_set(bn, "olqbar", bar);
        *has_mean = 2;
      }
    }
  } catch (std::exception& e) {
    err = e.what();
    return MGPU_ERR_ARGUMENT;
  }
  return MGPU_OK;
}

}  // namespace mgpu

extern "C" {

int mgpu_checkpoint_write_host(const mgpu_config* cfg, const char* path, const double* const* fields,
                               const double* mean, const mgpu_checkpoint_meta* meta) {
  if (!cfg || !path || !fields || !meta) return MGPU_ERR_ARGUMENT;
  mgpu::RefState rs;
  try {
    mgpu::build_reference_state(*cfg, rs);
  } catch (std::exception&) {
    return MGPU_ERR_ARGUMENT;
  }
  std::string err;
  int rc = mgpu::checkpoint_write_host(*cfg, rs, path, fields, mean, *meta, err);
  if (rc) std::fprintf(stderr, "mgpu_checkpoint_write_host: %s\n", err.c_str());
  return rc;
}

int mgpu_checkpoint_read_host(const mgpu_config* cfg, const char* path, double* const* fields, double* mean,
                              int32_t* has_mean, mgpu_checkpoint_meta* meta) {
  if (!cfg || !path || !fields || !meta) return MGPU_ERR_ARGUMENT;
  std::string err;
  int hm = 0;
  int rc = mgpu::checkpoint_read_host(*cfg, path, fields, mean, &hm, *meta, err);
  if (has_mean) *has_mean = hm;
  if (rc) std::fprintf(stderr, "mgpu_checkpoint_read_host: %s\n", err.c_str());
  return rc;
}

}  // extern "C"
