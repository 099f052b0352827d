// Run control around the step: the reference's input-file reader
// (LBM-C/infile_reader.cu), model builder (LBM-C/model_builder.cu), output
// handler (LBM-C/cgns/cgns_output_handler.cu) and driver loop
// (LBM-C/index.cu:61-153), as host C++ over the C ABI.  Host code only.
//
// Domain and output files: the reference reads and writes CGNS through a
// CGNS library that is not available to this build, so fields live in
// NumPy .npy files named after the reference's CGNS field names, and the
// output is a directory holding the same tree as the reference's CGNS file
// (index.json + one .npy per array).
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/lbmc.h"
#include "engine_internal.h"

namespace {

lbmc_status ferr(lbmc_status s, const std::string &m) {
  lbmc::set_last_error(m);
  return s;
}

void copy_str(char *dst, const std::string &s) {
  const size_t n = s.size() < LBMC_PATH_MAX - 1 ? s.size() : LBMC_PATH_MAX - 1;
  memcpy(dst, s.data(), n);
  dst[n] = 0;
}

template <class T>
std::string fmt(const T &v) {
  std::ostringstream o;
  o << v;
  return o.str();
}

// ------------------------------------------------------------ input file

// One line of an input file (the text before '#').  Keys are tried in the
// reference's order by substring; the first token is the name.
void input_line(const std::string &line, const std::string &whole, lbmc_run_config *rc, int &lz,
                int (&uz_flag), int (&node_z), std::string &echo) {
  std::istringstream ss(line);
  std::string name;
  auto has = [&](const char *k) { return line.find(k) != std::string::npos; };
  lbmc_config &c = rc->cfg;
  if (has("ProjName")) {
    std::string v;
    ss >> name >> v;
    copy_str(rc->project_name, v);
    echo += name + " = " + v + "\n";
  } else if (has("DomainFile")) {
    std::string v;
    ss >> name >> v;
    copy_str(rc->domain_file, v);
    echo += name + " = " + v + "\n";
  } else if (has("OutputFile")) {
    std::string v;
    ss >> name >> v;
    copy_str(rc->output_file, v);
    echo += name + " = " + v + "\n";
  } else if (has("TauMRT")) {
    ss >> name;
    int k = 0;
    double v;
    while (k < LBMC_MAX_Q && ss >> v) c.tau_mrt[k++] = v;
    rc->tau_mrt_count = k;
    for (int i = 0; i < k; i++) echo += "S_" + fmt(i) + " = " + fmt(c.tau_mrt[i]) + "\n";
  } else if (has("Tau")) {
    ss >> name >> c.tau;
    echo += name + " = " + fmt(c.tau) + "\n";
  } else if (has("Lx")) {
    ss >> name >> c.length[0];
    echo += name + " = " + fmt(c.length[0]) + "\n";
  } else if (has("Ly")) {
    ss >> name >> c.length[1];
    echo += name + " = " + fmt(c.length[1]) + "\n";
  } else if (has("Lz")) {
    ss >> name >> lz;
    rc->lz_given = 1;
    echo += name + " = " + fmt(lz) + "\n";
  } else if (has("DeltaX")) {
    ss >> name >> c.h;
    echo += name + " = " + fmt(c.h) + "\n";
  } else if (has("DeltaT")) {
    ss >> name >> c.dt;
    echo += name + " = " + fmt(c.dt) + "\n";
  } else if (has("C_smag")) {
    ss >> name >> c.c_smag;
    echo += name + " = " + fmt(c.c_smag) + "\n";
  } else if (has("ColType")) {
    // Each name found overrides the previous one, in this order, so
    // "MRTPOR" (which contains "MRT") ends as MRTPOR.
    std::string label;
    if (has("BGK")) { c.collision_type = LBMC_BGK; label = "BGK"; }
    if (has("NTPOR")) { c.collision_type = LBMC_NTPOR; label = "NTPOR"; }
    if (has("MRT")) { c.collision_type = LBMC_MRT; label = "MRT"; }
    if (has("MRTPOR")) { c.collision_type = LBMC_MRTPOR; label = "MRTPOR"; }
    ss >> name;
    echo += name + " = " + label + "\n";
  } else if (has("Force")) {
    int v = 0;
    ss >> name >> v;
    c.forcing = v != 0;
    echo += name + " = " + fmt(c.forcing) + "\n";
  } else if (has("MicroBC")) {
    int v = 0;
    ss >> name >> v;
    c.micro_bc = v != 0;
    echo += name + " = " + fmt(c.micro_bc) + "\n";
  } else if (has("MacroBC")) {
    int v = 0;
    ss >> name >> v;
    c.macro_bc = v != 0;
    echo += name + " = " + fmt(c.macro_bc) + "\n";
  } else if (has("Tolerance")) {
    ss >> name >> c.tolerance;
    echo += name + " = " + fmt(c.tolerance) + "\n";
  } else if (has("Init")) {
    ss >> name >> c.init_type;
    echo += name + " = " + fmt(c.init_type) + "\n";
  } else if (has("MaxT")) {
    ss >> name >> rc->max_t;
    echo += name + " = " + fmt(rc->max_t) + "\n";
  } else if (has("FileOut")) {
    ss >> name >> rc->file_out;
    echo += name + " = " + fmt(rc->file_out) + "\n";
  } else if (has("ScreenMes")) {
    ss >> name >> rc->screen_mes;
    echo += name + " = " + fmt(rc->screen_mes) + "\n";
  } else if (has("SteadyCheck")) {
    ss >> name >> rc->steady_check;
    echo += name + " = " + fmt(rc->steady_check) + "\n";
  } else if (has("OutputVars")) {
    int v[5] = {0, 0, 0, 0, 0};
    ss >> name >> v[0] >> v[1] >> v[2] >> v[3] >> v[4];
    rc->output_u[0] = v[0] != 0;
    rc->output_u[1] = v[1] != 0;
    uz_flag = v[2] != 0;
    rc->output_rho = v[3] != 0;
    rc->output_pressure = v[4] != 0;
    if (rc->output_u[0]) echo += "Output VelocityX = 1\n";
    if (rc->output_u[1]) echo += "Output VelocityY = 1\n";
    if (rc->output_rho) echo += "Output Density = 1\n";
    if (rc->output_pressure) echo += "Output Pressure = 1\n";
  } else if (has("ScreenNode")) {
    ss >> name >> rc->screen_node[0] >> rc->screen_node[1] >> node_z;
    echo += "Screen Node X = " + fmt(rc->screen_node[0]) + "\nScreen Node Y = " + fmt(rc->screen_node[1]) + "\n";
  } else if (has("Interactive")) {
    int v = 0;
    ss >> name >> v;
    rc->interactive = v != 0;
    echo += name + " = " + fmt(rc->interactive) + "\n";
  } else if (has("Lattice")) {
    std::string v;
    ss >> name >> v;
    if (v == "D3Q15" || v == "d3q15") c.lattice = LBMC_D3Q15;
    else c.lattice = LBMC_D2Q9;
    rc->lattice_given = 1;
    echo += name + " = " + v + "\n";
  } else {
    echo += whole + "\n";
  }
}

// ------------------------------------------------------------- .npy I/O

struct Npy {
  std::string descr;
  std::vector<long long> shape;
  std::vector<char> data;
  long long count() const {
    long long n = 1;
    for (long long s : shape) n *= s;
    return n;
  }
};

bool read_npy(const std::string &path, Npy &a, std::string &why) {
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    why = "cannot open " + path;
    return false;
  }
  char magic[8];
  in.read(magic, 8);
  if (!in || memcmp(magic, "\x93NUMPY", 6) != 0) {
    why = path + " is not a .npy file";
    return false;
  }
  size_t hlen = 0;
  if (magic[6] == 1) {
    unsigned char b[2];
    in.read(reinterpret_cast<char *>(b), 2);
    hlen = b[0] | (b[1] << 8);
  } else {
    unsigned char b[4];
    in.read(reinterpret_cast<char *>(b), 4);
    hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((size_t)b[3] << 24);
  }
  std::string h(hlen, ' ');
  in.read(&h[0], (std::streamsize)hlen);
  auto value_of = [&](const char *key) -> std::string {
    const size_t k = h.find(key);
    if (k == std::string::npos) return "";
    const size_t c = h.find(':', k);
    return c == std::string::npos ? "" : h.substr(c + 1);
  };
  std::string d = value_of("'descr'");
  const size_t q0 = d.find('\''), q1 = d.find('\'', q0 + 1);
  if (q0 == std::string::npos || q1 == std::string::npos) {
    why = path + ": no dtype in the header";
    return false;
  }
  a.descr = d.substr(q0 + 1, q1 - q0 - 1);
  const std::string fo = value_of("'fortran_order'");
  if (fo.find("True") != std::string::npos && fo.find("True") < fo.find(',')) {
    why = path + ": Fortran-ordered arrays are not supported";
    return false;
  }
  std::string sh = value_of("'shape'");
  const size_t p0 = sh.find('('), p1 = sh.find(')');
  a.shape.clear();
  std::istringstream ss(sh.substr(p0 + 1, p1 - p0 - 1));
  std::string tok;
  while (std::getline(ss, tok, ',')) {
    if (tok.find_first_not_of(" \t") == std::string::npos) continue;
    a.shape.push_back(std::stoll(tok));
  }
  size_t item = 0;
  if (a.descr == "<f8" || a.descr == "<i8") item = 8;
  else if (a.descr == "<f4" || a.descr == "<i4") item = 4;
  else if (a.descr == "|u1" || a.descr == "|i1") item = 1;
  else {
    why = path + ": unsupported dtype " + a.descr + " (float64/float32/int64/int32/uint8)";
    return false;
  }
  a.data.resize((size_t)a.count() * item);
  in.read(a.data.data(), (std::streamsize)a.data.size());
  if (!in) {
    why = path + ": file shorter than its header says";
    return false;
  }
  return true;
}

template <class T>
void npy_convert(const Npy &a, std::vector<T> &out) {
  const long long n = a.count();
  out.resize((size_t)n);
  const char *p = a.data.data();
  for (long long k = 0; k < n; k++) {
    if (a.descr == "<f8") { double v; memcpy(&v, p + 8 * k, 8); out[k] = (T)v; }
    else if (a.descr == "<f4") { float v; memcpy(&v, p + 4 * k, 4); out[k] = (T)v; }
    else if (a.descr == "<i8") { long long v; memcpy(&v, p + 8 * k, 8); out[k] = (T)v; }
    else if (a.descr == "<i4") { int v; memcpy(&v, p + 4 * k, 4); out[k] = (T)v; }
    else if (a.descr == "|u1") out[k] = (T)(unsigned char)p[k];
    else out[k] = (T)(signed char)p[k];
  }
}

bool write_npy(const std::string &path, const char *descr, const void *data, size_t item,
               const std::vector<long long> &shape) {
  std::string dict = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (";
  long long n = 1;
  for (size_t i = 0; i < shape.size(); i++) {
    dict += fmt(shape[i]) + (shape.size() == 1 || i + 1 < shape.size() ? ", " : "");
    n *= shape[i];
  }
  dict += "), }";
  size_t total = 10 + dict.size() + 1;
  const size_t pad = (64 - total % 64) % 64;
  dict += std::string(pad, ' ') + "\n";
  std::ofstream out(path, std::ios::binary);
  if (!out) return false;
  const unsigned short hl = (unsigned short)dict.size();
  out.write("\x93NUMPY\x01\x00", 8);
  const char hb[2] = {(char)(hl & 0xff), (char)(hl >> 8)};
  out.write(hb, 2);
  out.write(dict.data(), (std::streamsize)dict.size());
  out.write(static_cast<const char *>(data), (std::streamsize)(n * item));
  return (bool)out;
}

bool make_dir(const std::string &p) {
  if (mkdir(p.c_str(), 0755) == 0 || errno == EEXIST) return true;
  return false;
}

bool make_dirs(const std::string &p) {
  for (size_t k = 1; k <= p.size(); k++)
    if (k == p.size() || p[k] == '/')
      if (!make_dir(p.substr(0, k))) return false;
  return true;
}

std::string json_str(const std::string &s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}

}  // namespace

// ------------------------------------------------------------ input file

extern "C" lbmc_status lbmc_read_input(const char *path, lbmc_run_config *rc, char *echo, size_t echo_bytes) {
  if (!path || !rc) return ferr(LBMC_ERR_INVALID_ARG, "lbmc_read_input: NULL argument");
  std::ifstream in(path);
  if (!in) return ferr(LBMC_ERR_IO, std::string("lbmc_read_input: cannot open ") + path);
  memset(rc, 0, sizeof(*rc));
  lbmc_config_default(&rc->cfg, LBMC_D2Q9);
  rc->cfg.c_smag = 0;  // InfileReader::initialise
  rc->cfg.lattice = LBMC_D2Q9;
  int lz = 1, uz_flag = 0, node_z = 0;
  std::string echo_s, whole;
  while (std::getline(in, whole)) {
    std::string part = whole.substr(0, whole.find('#'));
    input_line(part, whole, rc, lz, uz_flag, node_z, echo_s);
  }
  if (!rc->lattice_given) rc->cfg.lattice = (rc->lz_given && lz > 1) ? LBMC_D3Q15 : LBMC_D2Q9;
  if (rc->cfg.lattice == LBMC_D3Q15) {
    rc->cfg.length[2] = lz;
    rc->output_u[2] = lz > 0 ? uz_flag : 0;
    rc->screen_node[2] = node_z;
    if (rc->output_u[2]) echo_s += "Output VelocityZ = 1\n";
    echo_s += "Screen Node Z = " + fmt(node_z) + "\n";
  } else {
    rc->cfg.length[2] = 1;
  }
  if (echo && echo_bytes) {
    const size_t n = echo_s.size() < echo_bytes - 1 ? echo_s.size() : echo_bytes - 1;
    memcpy(echo, echo_s.data(), n);
    echo[n] = 0;
  }
  return LBMC_OK;
}

// ----------------------------------------------------------- model build

struct lbmc_model {
  int dim = 2, q = 9;
  long long n = 0;
  std::vector<double> geometry, force[3], u[3], rho, f;
  std::vector<int> macro, micro;
};

extern "C" lbmc_status lbmc_model_build(const lbmc_run_config *rc, lbmc_model **out) {
  if (!rc || !out) return ferr(LBMC_ERR_INVALID_ARG, "lbmc_model_build: NULL argument");
  *out = nullptr;
  const lbmc_config &c = rc->cfg;
  auto m = new lbmc_model();
  m->dim = c.lattice == LBMC_D3Q15 ? 3 : 2;
  m->q = c.lattice == LBMC_D3Q15 ? 15 : 9;
  m->n = (long long)c.length[0] * c.length[1] * (m->dim == 3 ? c.length[2] : 1);
  if (m->n <= 0) {
    delete m;
    return ferr(LBMC_ERR_INVALID_ARG, "lbmc_model_build: Lx, Ly (and Lz) must be positive");
  }
  const std::string dir = rc->domain_file;
  std::string why;
  // Reads field `name` into dst (N values, or N * per values).
  auto load = [&](const char *name, auto &dst, bool required, long long per = 1) -> int {
    Npy a;
    const std::string p = dir + "/" + name + ".npy";
    struct stat st;
    if (stat(p.c_str(), &st) != 0) {
      if (required) why = std::string("domain field ") + name + " missing: " + p;
      return required ? -1 : 0;
    }
    if (!read_npy(p, a, why)) return -1;
    if (a.count() != m->n * per) {
      why = p + ": " + fmt(a.count()) + " values, expected " + fmt(m->n * per);
      return -1;
    }
    npy_convert(a, dst);
    return 1;
  };
  static const char *force_names[3] = {"ForceX", "ForceY", "ForceZ"};
  static const char *vel_names[3] = {"VelocityX", "VelocityY", "VelocityZ"};
  bool ok = load("Porosity", m->geometry, false) >= 0;
  if (ok && c.forcing)
    for (int d = 0; d < m->dim && ok; d++) ok = load(force_names[d], m->force[d], true) > 0;
  if (ok && c.micro_bc) ok = load("MicroBC", m->micro, true) > 0;
  const bool need_uv = c.macro_bc || c.init_type == LBMC_INIT_EQUILIBRIUM;
  if (ok && c.macro_bc) ok = load("MacroBC", m->macro, true) > 0;
  if (ok && need_uv) {
    for (int d = 0; d < m->dim && ok; d++) ok = load(vel_names[d], m->u[d], true) > 0;
    if (ok) ok = load("Rho", m->rho, true) > 0;
  }
  if (ok && c.init_type == LBMC_INIT_F) ok = load("Populations", m->f, true, m->q) > 0;
  if (!ok) {
    delete m;
    return ferr(LBMC_ERR_IO, "lbmc_model_build: " + why);
  }
  *out = m;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_model_domain(const lbmc_model *m, lbmc_domain *dom) {
  if (!m || !dom) return ferr(LBMC_ERR_INVALID_ARG, "lbmc_model_domain: NULL argument");
  memset(dom, 0, sizeof(*dom));
  auto ptr = [](const std::vector<double> &v) { return v.empty() ? nullptr : v.data(); };
  dom->geometry = ptr(m->geometry);
  for (int d = 0; d < 3; d++) {
    dom->force[d] = ptr(m->force[d]);
    dom->u[d] = ptr(m->u[d]);
  }
  dom->rho = ptr(m->rho);
  dom->f = ptr(m->f);
  dom->macro_bc = m->macro.empty() ? nullptr : m->macro.data();
  dom->micro_bc = m->micro.empty() ? nullptr : m->micro.data();
  return LBMC_OK;
}

extern "C" void lbmc_model_free(lbmc_model *m) { delete m; }

// --------------------------------------------------------------- output

struct lbmc_output {
  std::string path;
  int dim = 2;
  int L[3] = {1, 1, 1};
  std::vector<long long> steps;
  std::vector<std::string> solutions;
  std::vector<std::vector<std::string>> fields;
};

static bool write_index(const lbmc_output *o, bool closed) {
  const int nv[3] = {o->L[0] + 1, o->L[1] + 1, o->L[2] + 1};
  std::ostringstream j;
  j << "{\n \"format\": \"CGNS tree of the LBM-C output, arrays as .npy\",\n";
  j << " \"Base\": {\n  \"name\": \"Base\", \"cell_dim\": " << o->dim << ", \"phys_dim\": " << o->dim << ",\n";
  j << "  \"SimulationType\": \"TimeAccurate\",\n";
  j << "  \"BaseIterativeData\": {\"name\": \"TimeIterValues\", \"IterationValues\": [";
  for (size_t k = 0; k < o->steps.size(); k++) j << (k ? ", " : "") << o->steps[k];
  j << "]},\n";
  j << "  \"Zone\": {\n   \"name\": \"LBM-C Output Data\", \"type\": \"Structured\",\n";
  j << "   \"vertex_size\": [" << nv[0] << ", " << nv[1] << (o->dim == 3 ? ", " + fmt(nv[2]) : std::string()) << "],\n";
  j << "   \"cell_size\": [" << o->L[0] << ", " << o->L[1] << (o->dim == 3 ? ", " + fmt(o->L[2]) : std::string()) << "],\n";
  j << "   \"GridCoordinates\": {\"CoordinateX\": \"GridCoordinates/CoordinateX.npy\", "
       "\"CoordinateY\": \"GridCoordinates/CoordinateY.npy\""
    << (o->dim == 3 ? ", \"CoordinateZ\": \"GridCoordinates/CoordinateZ.npy\"" : "")
    << ", \"type\": \"RealSingle\"},\n";
  j << "   \"FlowSolutions\": [";
  for (size_t k = 0; k < o->solutions.size(); k++) {
    j << (k ? ",\n    " : "\n    ") << "{\"name\": " << json_str(o->solutions[k])
      << ", \"GridLocation\": \"CellCenter\", \"type\": \"RealDouble\", \"fields\": {";
    for (size_t f = 0; f < o->fields[k].size(); f++)
      j << (f ? ", " : "") << json_str(o->fields[k][f]) << ": "
        << json_str(o->solutions[k] + "/" + o->fields[k][f] + ".npy");
    j << "}}";
  }
  j << "],\n";
  j << "   \"ZoneIterativeData\": {\"FlowSolutionPointers\": [";
  for (size_t k = 0; k < o->solutions.size(); k++) j << (k ? ", " : "") << json_str(o->solutions[k]);
  j << "]}\n  }\n },\n \"complete\": " << (closed ? "true" : "false") << "\n}\n";
  std::ofstream out(o->path + "/index.json");
  out << j.str();
  return (bool)out;
}

extern "C" lbmc_status lbmc_output_open(const char *path, int dim, const int length[3], lbmc_output **out) {
  if (!path || !length || !out || (dim != 2 && dim != 3))
    return ferr(LBMC_ERR_INVALID_ARG, "lbmc_output_open: bad argument");
  auto o = new lbmc_output();
  o->path = path;
  o->dim = dim;
  for (int d = 0; d < 3; d++) o->L[d] = d < dim ? length[d] : 1;
  if (!make_dirs(o->path + "/GridCoordinates")) {
    delete o;
    return ferr(LBMC_ERR_IO, std::string("lbmc_output_open: cannot create ") + path);
  }
  // Vertex grid, coordinate = vertex index (cgns_output_handler.cu:74-154).
  const long long ni = o->L[0] + 1, nj = o->L[1] + 1, nk = dim == 3 ? o->L[2] + 1 : 1;
  std::vector<float> c(ni * nj * nk);
  const char *names[3] = {"CoordinateX", "CoordinateY", "CoordinateZ"};
  std::vector<long long> shape = dim == 3 ? std::vector<long long>{nk, nj, ni} : std::vector<long long>{nj, ni};
  for (int a = 0; a < dim; a++) {
    for (long long k = 0; k < nk; k++)
      for (long long j = 0; j < nj; j++)
        for (long long i = 0; i < ni; i++) c[i + ni * (j + nj * k)] = (float)(a == 0 ? i : a == 1 ? j : k);
    if (!write_npy(o->path + "/GridCoordinates/" + names[a] + ".npy", "<f4", c.data(), 4, shape)) {
      delete o;
      return ferr(LBMC_ERR_IO, std::string("lbmc_output_open: cannot write the grid under ") + path);
    }
  }
  write_index(o, false);
  *out = o;
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_output_append(lbmc_output *o, long long step, int nfields, const double *const *data,
                                          const char *const *labels) {
  if (!o || nfields < 0 || (nfields && (!data || !labels)))
    return ferr(LBMC_ERR_INVALID_ARG, "lbmc_output_append: bad argument");
  const std::string sol = "Solution @ Time = " + fmt(step);
  if (!make_dir(o->path + "/" + sol)) return ferr(LBMC_ERR_IO, "lbmc_output_append: cannot create " + sol);
  std::vector<long long> shape = o->dim == 3 ? std::vector<long long>{o->L[2], o->L[1], o->L[0]}
                                              : std::vector<long long>{o->L[1], o->L[0]};
  std::vector<std::string> names;
  for (int k = 0; k < nfields; k++) {
    if (!data[k] || !labels[k]) return ferr(LBMC_ERR_INVALID_ARG, "lbmc_output_append: NULL field");
    if (!write_npy(o->path + "/" + sol + "/" + labels[k] + ".npy", "<f8", data[k], 8, shape))
      return ferr(LBMC_ERR_IO, "lbmc_output_append: cannot write " + sol + "/" + labels[k]);
    names.push_back(labels[k]);
  }
  o->steps.push_back(step);
  o->solutions.push_back(sol);
  o->fields.push_back(names);
  write_index(o, false);
  return LBMC_OK;
}

extern "C" lbmc_status lbmc_output_close(lbmc_output *o) {
  if (!o) return LBMC_OK;
  const bool ok = write_index(o, true);
  const std::string p = o->path;
  delete o;
  if (!ok) return ferr(LBMC_ERR_IO, "lbmc_output_close: cannot write " + p + "/index.json");
  return LBMC_OK;
}

// ---------------------------------------------------------------- driver

namespace {

constexpr int NUM_RESIDS = 3;

struct Runner {
  lbmc_run_config rc;
  lbmc_model *model = nullptr;
  lbmc_handle *h = nullptr;
  lbmc_output *out = nullptr;
  bool quiet = false;
  int dim = 2;
  long long n = 0;
  std::vector<double> rho, u[3];
  ~Runner() {
    if (out) lbmc_output_close(out);
    if (h) lbmc_destroy(h);
    if (model) lbmc_model_free(model);
  }
  // output_macros (LBM-C/index.cu:196-281).
  lbmc_status output(long long t) {
    if (!out) return LBMC_OK;
    std::vector<const double *> data;
    std::vector<const char *> labels;
    static const char *vel[3] = {"VelocityX", "VelocityY", "VelocityZ"};
    for (int d = 0; d < dim; d++)
      if (rc.output_u[d]) {
        u[d].resize(n);
        lbmc_status s = lbmc_fetch(h, LBMC_FIELD_U_X + d, u[d].data(), n * sizeof(double));
        if (s != LBMC_OK) return s;
        data.push_back(u[d].data());
        labels.push_back(vel[d]);
      }
    if (rc.output_rho) {
      rho.resize(n);
      lbmc_status s = lbmc_fetch(h, LBMC_FIELD_RHO, rho.data(), n * sizeof(double));
      if (s != LBMC_OK) return s;
      data.push_back(rho.data());
      labels.push_back("Density");
    }
    lbmc_status s = lbmc_output_append(out, t, (int)data.size(), data.data(), labels.data());
    if (s == LBMC_OK && !quiet) printf("\nOutput Handler: Solution @ Time = %lld written\n", t);
    return s;
  }
};

}  // namespace

extern "C" lbmc_status lbmc_run(const char *input_path, const lbmc_config *ov, int quiet, lbmc_run_result *res) {
  if (!input_path || !res) return ferr(LBMC_ERR_INVALID_ARG, "lbmc_run: NULL argument");
  memset(res, 0, sizeof(*res));
  Runner r;
  r.quiet = quiet != 0;
  std::vector<char> echo(1 << 16);
  lbmc_status s = lbmc_read_input(input_path, &r.rc, echo.data(), echo.size());
  if (s != LBMC_OK) return s;
  if (!r.quiet) printf("\nReading configuration data: \n\n%s\nFinished reading configuration data.\n", echo.data());
  lbmc_config cfg = r.rc.cfg;
  if (ov) {
    cfg.storage = ov->storage;
    cfg.streaming = ov->streaming;
    cfg.device = ov->device;
    cfg.kernel = ov->kernel;
    cfg.storage_scale = ov->storage_scale;
    cfg.compat = ov->compat;
  }
  s = lbmc_model_build(&r.rc, &r.model);
  if (s != LBMC_OK) return s;
  lbmc_domain dom;
  lbmc_model_domain(r.model, &dom);
  s = lbmc_init(&cfg, &dom, &r.h);
  if (s != LBMC_OK) return s;
  r.dim = cfg.lattice == LBMC_D3Q15 ? 3 : 2;
  r.n = (long long)cfg.length[0] * cfg.length[1] * cfg.length[2];
  if (r.rc.output_file[0]) {
    s = lbmc_output_open(r.rc.output_file, r.dim, cfg.length, &r.out);
    if (s != LBMC_OK) return s;
  }
  if (!r.quiet) {
    printf("X-Length:\t\t%d\nY-Length:\t\t%d\n", cfg.length[0], cfg.length[1]);
    if (r.dim == 3) printf("Z-Length:\t\t%d\n", cfg.length[2]);
    printf("Relaxation Time (Tau):\t%f\n", cfg.tau);
  }
  const int plot = r.rc.file_out, screen = r.rc.screen_mes, steady = r.rc.steady_check;
  const long long maxT = r.rc.max_t;
  double residual[NUM_RESIDS];
  for (int k = 0; k < NUM_RESIDS; k++) residual[k] = 1.0;  // ModelBuilder::constant_loader
  double prev_ke = 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  auto due = [](long long i, int every) { return every > 0 && i % every == 0; };
  long long i = 0;
  while (i < maxT) {
    // Run straight to the next step that writes, prints or checks.
    long long next = maxT;
    for (int every : {plot, screen, steady})
      if (every > 0) {
        const long long k = (i / every + 1) * every;
        if (k < next) next = k;
      }
    const bool want_plot = due(next, plot), want_screen = due(next, screen), want_steady = due(next, steady);
    unsigned flags = LBMC_SYNC;
    if (want_plot || want_screen || want_steady) flags |= LBMC_STORE_MACROS;
    if (want_steady) flags |= LBMC_REDUCE_DIAG;
    s = lbmc_iterate(r.h, (int)(next - i), flags);
    i = next;
    if (s == LBMC_ERR_NAN) {
      // The reference writes an output and exits with 1 (index.cu:130-133).
      res->nonfinite = 1;
      res->steps = i;
      r.output(i);
      res->outputs = r.out ? (int)r.out->steps.size() : 0;
      break;
    }
    if (s != LBMC_OK) return s;
    if (want_plot) {
      s = r.output(i);
      if (s != LBMC_OK) return s;
    }
    if (want_steady) {
      lbmc_diag d;
      s = lbmc_fetch(r.h, LBMC_FIELD_DIAG, &d, sizeof(d));
      if (s != LBMC_OK) return s;
      // error_RMS (index.cu:377-385): relative change of the kinetic energy
      // per step over the check interval.
      const double ke = d.kinetic_energy;
      residual[i % NUM_RESIDS] = (std::fabs(ke - prev_ke) / steady) / ke;
      prev_ke = ke;
    }
    if (want_screen && !r.quiet) {
      const int *c = r.rc.screen_node;
      const long long node = c[0] + (long long)cfg.length[0] * (c[1] + (long long)cfg.length[1] * (r.dim == 3 ? c[2] : 0));
      double v[4] = {0, 0, 0, 0};
      if (node >= 0 && node < r.n) lbmc_probe(r.h, node, v);
      printf("time = %lld; rho = %g; uX = %g; uY = %g; ", i, v[0], v[1], v[2]);
      if (r.dim == 3) printf("uZ = %g; ", v[3]);
      printf("resid = %g\n", residual[i % NUM_RESIDS]);
    }
    if (want_steady) {
      int below = 0;
      for (int k = 0; k < NUM_RESIDS; k++) below += residual[k] < cfg.tolerance;
      if (std::isnan(residual[i % NUM_RESIDS])) {
        res->nonfinite = 1;
        res->steps = i;
        r.output(i);
        break;
      }
      if (below == NUM_RESIDS) {
        res->steady = 1;
        res->steps = i;
        if (!want_plot) {
          s = r.output(i);
          if (s != LBMC_OK) return s;
        }
        break;
      }
    }
    res->steps = i;
  }
  res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int k = 0; k < NUM_RESIDS; k++) res->residual[k] = residual[k];
  res->outputs = r.out ? (int)r.out->steps.size() : 0;
  if (!r.quiet) printf("\n\nTotal Run Time: %fs\n", res->seconds);
  return res->nonfinite ? LBMC_ERR_NAN : LBMC_OK;
}
