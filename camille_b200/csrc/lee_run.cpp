// lee_run: run a camille case (input deck, PLOT3D files, BC file, overset file) on the GPU
// through the C ABI of lee_b200.h, without the reference's MPI driver.
//
// Usage: lee_run <restart.q> [--deck camille.in] [--precision fp64|fp32c] [--parse-only]
//
// Like the reference's executable (src/core/main.cpp; simulation::initialize,
// src/core/simulation.cpp:28-246) it reads
//   - the input deck (inputDeck::parse_linesInputDeck, src/core/input.cpp:870-1000): '#' starts a
//     comment, a backslash joins a line to the next, each line splits on " =,;:\t" into a name
//     and a body, a later line of the same name replaces an earlier one; NAME's value is the
//     first body item and NAME KEYWORD's the item after KEYWORD (src/core/input.cpp:1060-1240);
//   - the PLOT3D grid, mean-flow function and restart solution (src/io/plot3d.cpp:183-989);
//   - the BC file (io::read_bc, src/io/io.cpp:957-1272): nine entries per line, a leading '-' on
//     an index counting from the block's last point;
//   - the Overture overset file (through lee_read_overset_file),
// then runs solver::solve (src/solver/solver.cpp:41-89): steps lastrun+1 .. NUM_TOTAL_TIMESTEP,
// under FIX_DT at DT, under FIX_CFL rescaling dt at every step by CFL / (the CFL of the previous
// dt), starting from the dummy 1e-6. At every REPORT_TIMESTEP-th step it prints the reference's
// line (io::report_timeadvancing, src/io/io.cpp:496-510), appends the min/max line to
// ./report/solution/solution (ReportSolution::minmax, :440-494) and writes camille.NNNNNN.q when
// io::write_solution_on_the_fly would (:850-877); camille.000000.q is the state read at start
// (src/core/simulation.cpp:224).
//
// One extension key, absent from the reference: SOURCE_MONOPOLE = x0, y0, z0, amplitude, omega,
// halfwidth, ramp_time (LEE_SOURCE_MONOPOLE). --parse-only prints what was read as one JSON
// line and uses no GPU.
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "lee_b200.h"

namespace {

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "lee_run: %s\n", msg.c_str());
  std::exit(1);
}

// ---------------------------------------------------------------------------------------------
// Input deck
// ---------------------------------------------------------------------------------------------

class Deck {
 public:
  explicit Deck(const std::string& path) {
    std::ifstream f(path);
    if (!f) die("cannot open the input deck " + path);
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(f, line)) {
      const size_t hash = line.find('#');
      if (hash != std::string::npos) line.erase(hash);
      lines.push_back(line);
    }
    // A backslash ends a line that continues on the next one; the character just before the
    // backslash is dropped with it, as the reference's merge does.
    for (size_t q = 0; q < lines.size(); ++q) {
      const size_t bs = lines[q].find('\\');
      if (bs == std::string::npos) continue;
      if (q + 1 == lines.size()) {
        lines[q].erase(bs);
      } else {
        lines[q + 1] = lines[q].substr(0, bs == 0 ? 0 : bs - 1) + lines[q + 1];
        lines[q].clear();
      }
    }
    for (const std::string& l : lines) {
      std::vector<std::string> tok;
      size_t a = 0;
      while (true) {
        a = l.find_first_not_of(kDelim, a);
        if (a == std::string::npos) break;
        const size_t b = l.find_first_of(kDelim, a);
        tok.push_back(l.substr(a, b == std::string::npos ? std::string::npos : b - a));
        if (b == std::string::npos) break;
        a = b;
      }
      if (tok.empty()) continue;
      entries_[tok[0]] = std::vector<std::string>(tok.begin() + 1, tok.end());
    }
  }

  bool has(const std::string& name) const { return entries_.count(name) != 0; }

  bool has(const std::string& name, const std::string& keyword) const {
    if (!has(name)) return false;
    const auto& b = body(name);
    for (size_t q = 0; q + 1 < b.size(); ++q)
      if (b[q] == keyword) return true;
    return false;
  }

  const std::vector<std::string>& body(const std::string& name) const {
    auto it = entries_.find(name);
    if (it == entries_.end()) die("the input deck has no " + name);
    return it->second;
  }

  std::string str(const std::string& name) const {
    const auto& b = body(name);
    if (b.empty()) die(name + " has no value");
    return b[0];
  }

  std::string str(const std::string& name, const std::string& keyword) const {
    const auto& b = body(name);
    for (size_t q = 0; q + 1 < b.size(); ++q)
      if (b[q] == keyword) return b[q + 1];
    die(name + " has no " + keyword);
  }

  int i(const std::string& n) const { return std::atoi(str(n).c_str()); }
  int i(const std::string& n, const std::string& k) const { return std::atoi(str(n, k).c_str()); }
  double d(const std::string& n) const { return std::atof(str(n).c_str()); }
  double d(const std::string& n, const std::string& k) const { return std::atof(str(n, k).c_str()); }

 private:
  static constexpr const char* kDelim = " =,;:\t\r";
  std::map<std::string, std::vector<std::string>> entries_;
};

// ---------------------------------------------------------------------------------------------
// PLOT3D whole-multiblock files: int32 counts, float64 data, i fastest
// ---------------------------------------------------------------------------------------------

// state slots: the five LEE slots, then the passive scalars of LEE_SCALAR (at most eight)
constexpr int kMaxSlots = 13;
int g_nv = 5;

struct Block {
  int n[3] = {1, 1, 1};
  long long N = 0;
  std::vector<double> xyz[3], mean[kMaxSlots], sol[kMaxSlots];
};

void read_ints(std::ifstream& f, int* dst, size_t n, const std::string& what) {
  if (n && !f.read(reinterpret_cast<char*>(dst), (std::streamsize)(n * 4))) die("short file " + what);
}

void read_doubles(std::ifstream& f, double* dst, size_t n, const std::string& what) {
  if (n && !f.read(reinterpret_cast<char*>(dst), (std::streamsize)(n * 8))) die("short file " + what);
}

std::vector<Block> read_grid(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) die("cannot open the grid file " + path);
  int nb = 0;
  read_ints(f, &nb, 1, path);
  if (nb < 1 || nb > 4096) die("grid file " + path + ": block count " + std::to_string(nb));
  std::vector<int> dims(3 * (size_t)nb);
  read_ints(f, dims.data(), dims.size(), path);
  std::vector<Block> blocks((size_t)nb);
  for (size_t b = 0; b < blocks.size(); ++b) {
    Block& k = blocks[b];
    for (int d = 0; d < 3; ++d) {
      k.n[d] = dims[3 * b + (size_t)d];
      if (k.n[d] < 1) die("grid file " + path + ": a dimension below 1");
    }
    k.N = (long long)k.n[0] * k.n[1] * k.n[2];
    for (int d = 0; d < 3; ++d) {
      k.xyz[d].resize((size_t)k.N);
      read_doubles(f, k.xyz[d].data(), (size_t)k.N, path);
    }
  }
  return blocks;
}

void read_mean(const std::string& path, std::vector<Block>& blocks) {
  std::ifstream f(path, std::ios::binary);
  if (!f) die("cannot open the mean-flow file " + path);
  int nb = 0;
  read_ints(f, &nb, 1, path);
  if (nb != (int)blocks.size()) die("mean-flow file " + path + ": block count differs from the grid's");
  std::vector<int> dims(4 * (size_t)nb);
  read_ints(f, dims.data(), dims.size(), path);
  for (size_t b = 0; b < blocks.size(); ++b) {
    for (int d = 0; d < 3; ++d)
      if (dims[4 * b + (size_t)d] != blocks[b].n[d]) die("mean-flow file " + path + ": dimensions differ");
    if (dims[4 * b + 3] != g_nv) die("mean-flow file " + path + ": " + std::to_string(g_nv) + " variables expected");
  }
  for (auto& k : blocks)
    for (int v = 0; v < g_nv; ++v) {
      k.mean[v].resize((size_t)k.N);
      read_doubles(f, k.mean[v].data(), (size_t)k.N, path);
    }
}

// The restart's step and time come from tau[2] and tau[3] (src/io/plot3d.cpp:775-780).
void read_solution(const std::string& path, std::vector<Block>& blocks, int* step, double* time) {
  std::ifstream f(path, std::ios::binary);
  if (!f) die("cannot open the restart file " + path);
  int nb = 0;
  read_ints(f, &nb, 1, path);
  if (nb != (int)blocks.size()) die("restart file " + path + ": block count differs from the grid's");
  std::vector<int> dims(3 * (size_t)nb);
  read_ints(f, dims.data(), dims.size(), path);
  for (size_t b = 0; b < blocks.size(); ++b)
    for (int d = 0; d < 3; ++d)
      if (dims[3 * b + (size_t)d] != blocks[b].n[d]) die("restart file " + path + ": dimensions differ");
  for (auto& k : blocks) {
    double tau[4];
    read_doubles(f, tau, 4, path);
    *step = (int)tau[2];
    *time = tau[3];
    for (int v = 0; v < g_nv; ++v) {
      k.sol[v].resize((size_t)k.N);
      read_doubles(f, k.sol[v].data(), (size_t)k.N, path);
    }
  }
}

// tau = {0, 1, step, time} (src/io/plot3d.cpp:1289). With more than five slots (LEE_SCALAR) the
// reference writes the PLOT3D function format instead: (nxi, neta, nzeta, nvar) per block and no
// tau (io::write_solution, src/io/io.cpp:740-760); it still reads restarts as solution files.
void write_solution(const std::string& path, const std::vector<Block>& blocks, int step, double time) {
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) die("cannot write " + path);
  const int nb = (int)blocks.size();
  const bool function_form = g_nv != 5;
  f.write(reinterpret_cast<const char*>(&nb), 4);
  for (auto& k : blocks) {
    f.write(reinterpret_cast<const char*>(k.n), 12);
    if (function_form) f.write(reinterpret_cast<const char*>(&g_nv), 4);
  }
  for (auto& k : blocks) {
    const double tau[4] = {0.0, 1.0, (double)step, time};
    if (!function_form) f.write(reinterpret_cast<const char*>(tau), 32);
    for (int v = 0; v < g_nv; ++v)
      f.write(reinterpret_cast<const char*>(k.sol[v].data()), (std::streamsize)(k.N * 8));
  }
  if (!f) die("short write to " + path);
}

// ---------------------------------------------------------------------------------------------
// BC file
// ---------------------------------------------------------------------------------------------

struct BcLine {
  int block, kind, dir, end, lo[3], hi[3];
};

// io::parse_boundary_type (src/io/io.cpp:1275-1320) for the kinds the library implements.
int bc_kind(const std::string& s) {
  if (s == "dirichlet_allzero") return LEE_BC_DIRICHLET_ALLZERO;
  if (s == "dirichlet_harmonicwave") return LEE_BC_DIRICHLET_HARMONICWAVE;
  if (s == "neumann") return LEE_BC_NEUMANN;
  if (s == "wall_slip_kinematic") return LEE_BC_WALL_SLIP_KINEMATIC;
  if (s == "centerline_cart_norm2x") return LEE_BC_CENTERLINE_CART_NORM2X;
  if (s == "centerline_cart_norm2y") return LEE_BC_CENTERLINE_CART_NORM2Y;
  if (s == "centerline_cart_norm2z") return LEE_BC_CENTERLINE_CART_NORM2Z;
  if (s == "centerline_axisym") return LEE_BC_CENTERLINE_AXISYM;
  if (s == "sponge_freund_ambient") return LEE_SPONGE_FREUND_AMBIENT;
  if (s == "sponge_freund_harmonicwave") return LEE_SPONGE_FREUND_HARMONICWAVE;
  die("boundary type " + s + " is not implemented by the library");
}

std::string lower(std::string s) {
  for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

int bc_index(const std::string& e, int npoints) {
  const bool from_end = e[0] == '-';
  const int v = std::atoi((e[0] == '+' || e[0] == '-') ? e.c_str() + 1 : e.c_str());
  return from_end ? (npoints - 1) - v : v;
}

std::vector<BcLine> read_bc(const std::string& path, const std::vector<Block>& blocks) {
  std::ifstream f(path);
  if (!f) die("cannot open the BC file " + path);
  std::vector<BcLine> out;
  std::string line;
  while (std::getline(f, line)) {
    std::stringstream ss(line);
    std::vector<std::string> e;
    std::string w;
    while (ss >> w) e.push_back(w);
    if (e.empty() || e[0][0] == '#') continue;  // empty, blank or comment line
    for (const auto& x : e)
      if (x[0] == '#') die("BC file: an entry starts with a comment sign: " + line);
    if (e.size() != 9) die("BC file: nine entries expected: " + line);
    BcLine b{};
    b.block = std::atoi(e[0].c_str());
    if (b.block < 0 || b.block >= (int)blocks.size()) die("BC file: block index: " + line);
    b.kind = bc_kind(e[1]);
    if (e[2][0] == '+') b.end = 0;
    else if (e[2][0] == '-') b.end = 1;
    else die("BC file: unknown side: " + line);
    const std::string dn = lower(e[2].substr(1));
    b.dir = dn == "xi" ? 0 : dn == "eta" ? 1 : dn == "zeta" ? 2 : -1;
    if (b.dir < 0) die("BC file: unknown direction: " + line);
    for (int d = 0; d < 3; ++d) {
      b.lo[d] = bc_index(e[(size_t)(3 + 2 * d)], blocks[(size_t)b.block].n[d]);
      b.hi[d] = bc_index(e[(size_t)(4 + 2 * d)], blocks[(size_t)b.block].n[d]);
    }
    out.push_back(b);
  }
  return out;
}

// ---------------------------------------------------------------------------------------------
// Solver configuration from the deck (UserInput::set_inputDeck, src/core/input.cpp:99-284)
// ---------------------------------------------------------------------------------------------

struct Run {
  lee_config cfg{};
  std::string fix, simulation, overset = "NONE", grid, mean, bc, overset_file;
  double dt = 0.0, cfl = 0.0, writing_time = 0.0;
  int num_time_steps = 0, report_freq = 1, overset_order = 0;
  bool has_monopole = false;
  double monopole[7] = {};
  bool axisym = false;
  bool jet2d = false;  // SIMULATION = CASE_2DJET_WITH_A_HARMONIC_SOURCE
  // HARMONIC_WAVE (type LEE_WAVE_NONE when the deck says NONE)
  int wave_type = LEE_WAVE_NONE, wave_form = -1, wave_dir = 0;
  double wave_amp = 0.0, wave_len = 0.0, wave_hw = 0.0;
  int nsc = 0;  // PHYSICAL_MODEL = LEE_SCALAR: NUMBER_SCALAR
};

Run configure(const Deck& d, int precision) {
  Run r;
  const std::string model = d.str("PHYSICAL_MODEL");
  if (model == "LEE_SCALAR") {
    // src/core/input.cpp:113-117, and check_consistency_simulation (:596-606): LEE_SCALAR runs the
    // linear nozzle only
    r.nsc = d.i("PHYSICAL_MODEL", "NUMBER_SCALAR");
    if (!(r.nsc >= 1)) die("For PHYSICAL_MODEL = " + model + ", at least one scalar should be solved for.");
    if (r.nsc > kMaxSlots - 5) die("NUMBER_SCALAR above " + std::to_string(kMaxSlots - 5));
    if (d.str("SIMULATION") != "CASE_LINEAR_NOZZLE")
      die("SIMULATION " + d.str("SIMULATION") + " is not implemented for PHYSICAL_MODEL = " + model + ".");
  } else if (model != "LEE") {
    die("PHYSICAL_MODEL " + model + ": the library runs LEE and LEE_SCALAR");
  }
  g_nv = 5 + r.nsc;
  std::string axisym = d.has("AXISYMMETRY") ? d.str("AXISYMMETRY") : "FALSE";
  for (auto& ch : axisym) ch = (char)std::toupper((unsigned char)ch);  // truefalse_2int (:786-799)
  if (axisym == "TRUE") {
    // src/core/input.cpp:105-108 and check_consistency_dimension (:519-535)
    std::string axis = d.str("AXISYMMETRY", "AXIS_OF_SYMMETRY");
    for (auto& ch : axis) ch = (char)std::toupper((unsigned char)ch);
    if (axis != "X" && axis != "Y" && axis != "R" && axis != "Z") die("AXIS_OF_SYMMETRY " + axis);
    if (d.i("DIMENSION") != 2) die("Axisymmetry requires 2-D.");
    if (axis != "X") die("The axis of symmetry should be x by definition of the coordinate system.");
    r.axisym = true;
  } else if (axisym != "FALSE") {
    die("AXISYMMETRY " + axisym);
  }
  if (d.has("HARMONIC_WAVE") && d.str("HARMONIC_WAVE") != "NONE") {
    // src/core/input.cpp:219-231, then check_consistency_wave (:629-656), whose else clauses
    // bind to the inner ifs: only an acoustic wave of another shape and the amplitude range
    // stop the run there; a type or shape without a formula stops it at the first boundary
    // update that evaluates the wave (src/solver/boundary_condition.cpp:263-307)
    const std::string type = d.str("HARMONIC_WAVE"), form = d.str("HARMONIC_WAVE", "SHAPE");
    r.wave_amp = d.d("HARMONIC_WAVE", "AMPLITUDE");
    std::string dir = d.str("HARMONIC_WAVE", "DIRECTION");
    for (auto& ch : dir) ch = (char)std::toupper((unsigned char)ch);
    r.wave_dir = dir == "X" ? 0 : (dir == "Y" || dir == "R") ? 1 : dir == "Z" ? 2 : -1;
    if (r.wave_dir < 0) die("HARMONIC_WAVE DIRECTION " + dir);
    r.wave_len = d.d("HARMONIC_WAVE", "WAVELENGTH");
    if (form == "WAVEFORM_GAUSSIAN_ROUNDJET") r.wave_hw = d.d("HARMONIC_WAVE", "HALFWIDTH");
    if (type == "WAVE_ACOUSTIC" && form != "WAVEFORM_PLANE" && form != "WAVEFORM_HOMOGENEOUS")
      die("Unknown spatial distribution of acoustic waves.");
    if (r.wave_amp < 0.0 || r.wave_amp > 1.0) die("The wave amplitude should be between 0 and 1.");
    r.wave_type = type == "WAVE_ACOUSTIC" ? LEE_WAVE_ACOUSTIC : type == "WAVE_ENTROPY" ? LEE_WAVE_ENTROPY : -1;
    r.wave_form = form == "WAVEFORM_PLANE"           ? LEE_WAVEFORM_PLANE
                  : form == "WAVEFORM_HOMOGENEOUS"   ? LEE_WAVEFORM_HOMOGENEOUS
                  : form == "WAVEFORM_GAUSSIAN_ROUNDJET" ? LEE_WAVEFORM_GAUSSIAN_ROUNDJET
                                                     : -1;
  }
  if (d.has("INTERPOLATE_SOLUTION") && d.str("INTERPOLATE_SOLUTION") != "NONE")
    die("INTERPOLATE_SOLUTION is a pre-processing mode, not a time advance");
  if (d.has("FILE_FORMAT") && d.str("FILE_FORMAT") != "PLOT3D") die("FILE_FORMAT " + d.str("FILE_FORMAT"));
  if (d.has("METRIC_SCHEME") && d.str("METRIC_SCHEME") != "THOMAS_LOMBARD") die("METRIC_SCHEME " + d.str("METRIC_SCHEME"));
  lee_config& c = r.cfg;
  c.num_dim = d.i("DIMENSION");
  if (c.num_dim != 2 && c.num_dim != 3) die("DIMENSION is 2 or 3");
  c.gamma = d.d("GAMMA_SPECIFICHEAT");
  c.precision = precision;
  // physical source by case (source::apply_physicalSource, src/solver/source.cpp:22-107)
  r.simulation = d.has("SIMULATION") ? d.str("SIMULATION") : "NONE";
  // the 2-D jet's harmonic pressure source (src/solver/source.cpp:27-58): LEE_SOURCE_JET2D_HARMONIC
  r.jet2d = r.simulation == "CASE_2DJET_WITH_A_HARMONIC_SOURCE";
  if (r.simulation == "CASE_SCATTERING_TWOCYLINDER") {
    // (gamma - 1) exp(-ln 2 r^2 / 0.2^2) sin(4 2pi t), ramped by sin^2(pi t / 8) up to t = 4
    // (src/solver/source.cpp:60-92): the library's monopole at the origin.
    const double p[7] = {0.0, 0.0, 0.0, 1.0, 4.0 * (2.0 * M_PI), 0.2, 16.0 / 4.0};
    std::copy(p, p + 7, r.monopole);
    r.has_monopole = true;
  }
  if (d.has("SOURCE_MONOPOLE")) {
    const auto& b = d.body("SOURCE_MONOPOLE");
    if (b.size() != 7) die("SOURCE_MONOPOLE takes x0, y0, z0, amplitude, omega, halfwidth, ramp_time");
    for (int q = 0; q < 7; ++q) r.monopole[q] = std::atof(b[(size_t)q].c_str());
    r.has_monopole = true;
    if (r.jet2d) die("SOURCE_MONOPOLE does not combine with the source of CASE_2DJET_WITH_A_HARMONIC_SOURCE");
  }
  // time advance (src/core/input.cpp:129-139)
  r.fix = d.str("FIX_DT_OR_CFL");
  if (r.fix == "FIX_DT") r.dt = d.d("DT");
  else if (r.fix == "FIX_CFL") r.cfl = d.d("CFL");
  else die("You may fix either DT or CFL in time integration.");
  const std::string rk = d.str("TEMPORAL_SCHEME");
  c.rk_scheme = rk == "RUNGE_KUTTA4" ? LEE_RK4 : rk == "RUNGE_KUTTA2" ? LEE_RK2 : -1;
  if (c.rk_scheme < 0) die("TEMPORAL_SCHEME " + rk);
  r.num_time_steps = d.i("NUM_TOTAL_TIMESTEP");
  r.report_freq = d.i("REPORT_TIMESTEP");
  if (r.report_freq < 1) die("REPORT_TIMESTEP must be positive");
  // spatial operators (src/core/input.cpp:142-167)
  const std::string fd = d.str("SPATIAL_SCHEME");
  if (fd == "STANDARD_CENTRAL") {
    c.fd_scheme = LEE_FD_STANDARD_CENTRAL;
    c.fd_order = d.i("SPATIAL_SCHEME", "ORDER_ACCURACY");
  } else if (fd == "FDO11P") {
    c.fd_scheme = LEE_FD_FDO11P;
  } else {
    die("SPATIAL_SCHEME " + fd);
  }
  const std::string fl = d.str("SPATIAL_FILTER");
  c.filter_strength = 1.0;
  c.filter_blend = 1.0;
  if (fl == "NONE") {
    c.filter_scheme = LEE_FILTER_NONE;
  } else {
    if (fl == "STANDARD_CENTRAL") {
      c.filter_scheme = LEE_FILTER_STANDARD_CENTRAL;
      c.filter_order = d.i("SPATIAL_FILTER", "ORDER_ACCURACY");
    } else if (fl == "SFO11P") {
      c.filter_scheme = LEE_FILTER_SFO11P;
      c.filter_strength = d.d("SPATIAL_FILTER", "STRENGTH");
    } else {
      die("SPATIAL_FILTER " + fl);
    }
    c.filter_blend = d.d("SPATIAL_FILTER", "BLEND");
  }
  c.sponge_order = d.i("BUFFER_ZONE", "POLYNOMIAL_ORDER");
  c.sponge_constant = d.d("BUFFER_ZONE", "CONSTANT");
  // files (src/core/input.cpp:173-217)
  r.overset = d.str("OVERSET");
  if (r.overset != "NONE") {
    if (r.overset != "OVERTURE") die("OVERSET " + r.overset + ": the library reads Overture files");
    if (d.has("OVERSET", "TYPE") && d.str("OVERSET", "TYPE") != "EXPLICIT") die("OVERSET TYPE " + d.str("OVERSET", "TYPE"));
    r.overset_order = d.i("OVERSET", "ORDER_ACCURACY");
    r.overset_file = d.str("OVERSET_FILE");
  }
  r.grid = d.str("GRID_FILE");
  r.mean = d.str("BASESTATE_FILE");
  r.bc = d.str("BC_FILE");
  r.writing_time = d.has("SOLUTION_WRITING_TIME") ? d.d("SOLUTION_WRITING_TIME") : 1e300;
  return r;
}

void check(lee_ctx* c, int rc, const char* what) {
  if (rc != LEE_OK) die(std::string(what) + ": " + lee_last_error(c));
}

std::string solution_name(int counter) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "camille.%06d.q", counter);
  return buf;
}

void print_parse(const Run& r, const std::vector<Block>& blocks, const std::vector<BcLine>& bcs, int step, double time) {
  const lee_config& c = r.cfg;
  std::printf("{\"num_dim\": %d, \"gamma\": %.17g, \"blocks\": [", c.num_dim, c.gamma);
  for (size_t b = 0; b < blocks.size(); ++b)
    std::printf("%s[%d, %d, %d]", b ? ", " : "", blocks[b].n[0], blocks[b].n[1], blocks[b].n[2]);
  std::printf("], \"fd\": [%d, %d], \"filter\": [%d, %d, %.17g, %.17g], \"rk\": %d, \"sponge\": [%d, %.17g], "
              "\"fix\": \"%s\", \"dt\": %.17g, \"cfl\": %.17g, \"num_time_steps\": %d, \"report\": %d, "
              "\"writing_time\": %.17g, \"step\": %d, \"time\": %.17g, \"overset\": \"%s\", \"overset_order\": %d, "
              "\"monopole\": ",
              c.fd_scheme, c.fd_order, c.filter_scheme, c.filter_order, c.filter_strength, c.filter_blend, c.rk_scheme,
              c.sponge_order, c.sponge_constant, r.fix.c_str(), r.dt, r.cfl, r.num_time_steps, r.report_freq,
              r.writing_time, step, time, r.overset.c_str(), r.overset_order);
  if (r.has_monopole) {
    std::printf("[");
    for (int q = 0; q < 7; ++q) std::printf("%s%.17g", q ? ", " : "", r.monopole[q]);
    std::printf("]");
  } else {
    std::printf("null");
  }
  std::printf(", \"wave\": [%d, %d, %d, %.17g, %.17g, %.17g], \"axisym\": %s, \"jet2d\": %s", r.wave_type,
              r.wave_form, r.wave_dir, r.wave_amp, r.wave_len, r.wave_hw, r.axisym ? "true" : "false",
              r.jet2d ? "true" : "false");
  std::printf(", \"scalars\": %d", r.nsc);
  std::printf(", \"bc\": [");
  for (size_t q = 0; q < bcs.size(); ++q)
    std::printf("%s[%d, %d, %d, %d, %d, %d, %d, %d, %d, %d]", q ? ", " : "", bcs[q].block, bcs[q].kind, bcs[q].dir,
                bcs[q].end, bcs[q].lo[0], bcs[q].hi[0], bcs[q].lo[1], bcs[q].hi[1], bcs[q].lo[2], bcs[q].hi[2]);
  std::printf("]}\n");
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2 || argv[1][0] == '-')
    die("usage: lee_run <restart.q> [--deck camille.in] [--precision fp64|fp32c] [--parse-only]");
  const std::string restart = argv[1];
  std::string deck_path = "camille.in";
  int precision = LEE_FP64;
  bool parse_only = false;
  for (int a = 2; a < argc; ++a) {
    const std::string s = argv[a];
    if (s == "--deck" && a + 1 < argc) {
      deck_path = argv[++a];
    } else if (s == "--precision" && a + 1 < argc) {
      const std::string p = argv[++a];
      if (p == "fp64") precision = LEE_FP64;
      else if (p == "fp32c") precision = LEE_FP32_COMPENSATED;
      else die("--precision is fp64 or fp32c");
    } else if (s == "--parse-only") {
      parse_only = true;
    } else {
      die("unknown argument " + s);
    }
  }
  const Deck deck(deck_path);
  Run r = configure(deck, precision);
  std::vector<Block> blocks = read_grid(r.grid);
  read_mean(r.mean, blocks);
  int step = 0;
  double time = 0.0;
  read_solution(restart, blocks, &step, &time);
  const std::vector<BcLine> bcs = read_bc(r.bc, blocks);
  r.cfg.num_blocks = (int)blocks.size();
  if (parse_only) {
    print_parse(r, blocks, bcs, step, time);
    return 0;
  }

  lee_ctx* c = nullptr;
  if (lee_create(&r.cfg, &c) != LEE_OK) die(std::string("lee_create: ") + lee_last_error(nullptr));
  if (r.nsc) check(c, lee_set_scalars(c, r.nsc), "NUMBER_SCALAR");
  for (size_t b = 0; b < blocks.size(); ++b) {
    Block& k = blocks[b];
    check(c, lee_set_block(c, (int)b, k.n[0], k.n[1], k.n[2], k.xyz[0].data(), k.xyz[1].data(), k.xyz[2].data(), nullptr),
          "grid");
    const double* m[5] = {k.mean[0].data(), k.mean[1].data(), k.mean[2].data(), k.mean[3].data(), k.mean[4].data()};
    check(c, lee_set_mean(c, (int)b, m), "mean flow");
    if (r.nsc) {
      const double* zm[kMaxSlots];
      for (int q = 0; q < r.nsc; ++q) zm[q] = k.mean[5 + q].data();
      check(c, lee_set_mean_scalars(c, (int)b, zm), "mean scalars");
    }
  }
  for (const BcLine& b : bcs) check(c, lee_add_boundary(c, b.block, b.kind, b.dir, b.end, b.lo, b.hi, nullptr), "BC file");
  bool wave_lines = false;
  for (const BcLine& b : bcs)
    wave_lines |= b.kind == LEE_BC_DIRICHLET_HARMONICWAVE || b.kind == LEE_SPONGE_FREUND_HARMONICWAVE;
  if (wave_lines) {
    // the reference reads the wave only where a line evaluates it
    if (r.wave_type == LEE_WAVE_NONE) die("Unknown type of wave form.");
    if (r.wave_type < 0 || r.wave_form < 0) die("Unknown type of wave for this wave form.");
    check(c, lee_set_harmonic_wave(c, r.wave_type, r.wave_form, r.wave_dir, r.wave_amp, r.wave_len, r.wave_hw),
          "HARMONIC_WAVE");
  }
  if (r.axisym) check(c, lee_set_axisymmetric(c, 1, 0), "AXISYMMETRY");
  if (r.has_monopole) check(c, lee_set_source(c, LEE_SOURCE_MONOPOLE, r.monopole, 7), "source");
  if (r.jet2d) check(c, lee_set_source(c, LEE_SOURCE_JET2D_HARMONIC, nullptr, 0), "source");
  if (r.overset != "NONE") check(c, lee_read_overset_file(c, r.overset_file.c_str(), r.overset_order), "overset file");
  check(c, lee_prepare(c), "lee_prepare");
  for (size_t b = 0; b < blocks.size(); ++b) {
    const double* s[5] = {blocks[b].sol[0].data(), blocks[b].sol[1].data(), blocks[b].sol[2].data(),
                          blocks[b].sol[3].data(), blocks[b].sol[4].data()};
    check(c, lee_upload_state(c, (int)b, s, step, time), "restart");
    if (r.nsc) {
      const double* z[kMaxSlots];
      for (int q = 0; q < r.nsc; ++q) z[q] = blocks[b].sol[5 + q].data();
      check(c, lee_upload_scalars(c, (int)b, z), "restart scalars");
    }
  }

  int counter = 0;
  write_solution(solution_name(counter), blocks, step, time);
  ::mkdir("report", 0755);
  ::mkdir("report/solution", 0755);
  static const char* kNames[5] = {"S'", "UX'", "UY'", "UZ'", "P'"};

  // The CFL of a dt is a fixed function of dt (the mean flow does not change): memoised, so that
  // FIX_CFL's sequence of dts, which settles within a few steps, costs one reduction per new dt.
  std::map<double, double> cfl_of;
  auto cfl_at = [&](double dt) {
    auto it = cfl_of.find(dt);
    if (it != cfl_of.end()) return it->second;
    double v = 0.0;
    check(c, lee_compute_cfl(c, dt, &v), "lee_compute_cfl");
    cfl_of[dt] = v;
    return v;
  };
  const int lastrun = step;
  const double time_lastrun = time;
  double dt = r.fix == "FIX_DT" ? r.dt : 1e-6;  // FIX_CFL starts from the dummy dt (src/core/input.cpp:131)
  int s = lastrun + 1;
  while (s <= r.num_time_steps) {
    // one run of steps with the same dt, ending at the next report step at the latest
    double cfl_max = cfl_at(dt);
    double dt_run = dt;
    if (r.fix == "FIX_CFL") dt_run = dt * (r.cfl / cfl_max);
    int e = s;
    const int next_report = ((s + r.report_freq - 1) / r.report_freq) * r.report_freq;
    const int last = std::min(r.num_time_steps, next_report);
    double report_cfl = cfl_max;
    if (r.fix == "FIX_CFL") {
      double cur = dt_run;
      while (e < last) {
        const double cm = cfl_at(cur);
        const double nxt = cur * (r.cfl / cm);
        if (nxt != dt_run) break;
        report_cfl = cm;
        cur = nxt;
        ++e;
      }
    } else {
      e = last;
    }
    check(c, lee_advance(c, e - s + 1, dt_run), "lee_advance");
    for (int q = s; q <= e; ++q) time += dt_run;  // time_sol += dt of every step, as the library's block clocks
    dt = dt_run;
    s = e + 1;
    if (e % r.report_freq == 0) {
      std::printf("Time step: %10d, time: %e, dt: %e, CFL: %e\n", e, time, dt, report_cfl);
      double mn[5], mx[5];
      check(c, lee_state_minmax(c, mn, mx), "lee_state_minmax");
      FILE* f = std::fopen("report/solution/solution", "a");
      if (!f) die("cannot append to report/solution/solution");
      std::fprintf(f, "Time step: %10d, time: %e", e, time);
      for (int v = 0; v < 5; ++v) std::fprintf(f, ", %s: %e ~ %e", kNames[v], mn[v], mx[v]);
      if (r.nsc) {
        // the scalar slots over every point of every block; their names grow as
        // State::initialize_state_linearizedEuler_scalar builds them with one stringstream
        // (src/core/state.cpp:350-357): Z0', Z01', Z012', ...
        std::string digits;
        for (int q = 0; q < r.nsc; ++q) {
          double lo = HUGE_VAL, hi = -HUGE_VAL;
          for (size_t b = 0; b < blocks.size(); ++b) {
            if (q == 0) {
              double* z[kMaxSlots];
              for (int w = 0; w < r.nsc; ++w) z[w] = blocks[b].sol[5 + w].data();
              check(c, lee_download_scalars(c, (int)b, z), "lee_download_scalars");
            }
            for (double v : blocks[b].sol[5 + q]) {
              lo = std::min(lo, v);
              hi = std::max(hi, v);
            }
          }
          digits += std::to_string(q);
          std::fprintf(f, ", Z%s': %e ~ %e", digits.c_str(), lo, hi);
        }
      }
      std::fprintf(f, "\n");
      std::fclose(f);
      const bool by_time = (int)((time - time_lastrun) / r.writing_time) > counter;
      if (by_time || e == r.num_time_steps) {
        ++counter;
        for (size_t b = 0; b < blocks.size(); ++b) {
          double* sol[5] = {blocks[b].sol[0].data(), blocks[b].sol[1].data(), blocks[b].sol[2].data(),
                            blocks[b].sol[3].data(), blocks[b].sol[4].data()};
          check(c, lee_download_state(c, (int)b, sol, &step, nullptr), "lee_download_state");
          if (r.nsc) {
            double* z[kMaxSlots];
            for (int q = 0; q < r.nsc; ++q) z[q] = blocks[b].sol[5 + q].data();
            check(c, lee_download_scalars(c, (int)b, z), "lee_download_scalars");
          }
        }
        write_solution(solution_name(counter), blocks, step, time);
      }
    }
  }
  lee_destroy(c);
  return 0;
}
