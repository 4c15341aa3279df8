// `.fdtd` script front-end with TetFIT's semantics: the DEFINE/SET/END line
// parser (src/DGA/Discretization.hpp:45-211), the primitive setters
// (Material.hpp:45-316, BoundaryCondition.hpp:45-125, Source.hpp:60-300,
// Output.hpp:58-298, Simulation.hpp:52-97, Mesh.hpp:44-251, Solid.hpp:44-262)
// and the solids-file reader (Discretization.hpp:4219-4345).
//
// Parity notes (documented divergences, all in undefined-behaviour corners of
// the reference): token buffers are larger than the reference's 10/20/64
// char arrays; a `bc` surface label >= 100 is rejected instead of writing past
// the 100-slot BndToBC table (Discretization.hpp:61,119-128).
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace tf {

// Utilities.hpp:92-95.  PI is a long double literal there; mu0 is evaluated in
// long double and stored as double.
const long double PI_L = 3.141592653589793238L;
const double MU0 = (double)(4 * PI_L * 1e-7);
const double EPS0 = 8.854187817e-12;
const double C0 = 1 / std::sqrt(MU0 * EPS0);

struct ScriptError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// Utilities.hpp:371-375: "Input file error at line N: <msg>".
[[noreturn]] void my_throw(uint32_t line, const std::string& msg);

struct Mat3 {  // diagonal-or-full 3x3, row-major
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  static Mat3 diag(double d) {
    Mat3 r;
    r.m[0][0] = r.m[1][1] = r.m[2][2] = d;
    return r;
  }
};

struct Material {  // Material.hpp:37-51
  Mat3 eps = Mat3::diag(EPS0), mu = Mat3::diag(MU0), sigma, chi;
  void set(uint32_t line, const std::string& p, const std::string& v);
};

struct BoundaryCondition {  // BoundaryCondition.hpp:37-44
  std::string type = "none", dir = "none";
  double width = 0, val = 0;
  std::vector<uint32_t> surfs;
  void set(uint32_t line, const std::string& p, const std::string& v);
};

struct Source {  // Source.hpp:37-57
  std::string st = " ", prof = "dc", carrier = "sin", dir = "x";
  double amp = 0, freq = 0, radius = 1, decay = 0, width = 1, delay = 0, impedance = 50;
  std::array<double, 3> kvec{0, 0, 0}, center{0, 0, 0}, location{0, 0, 0};
  std::array<std::string, 3> bfuncs{"cos", "cos", "cos"};
  std::vector<uint32_t> surfaces;
  void set(uint32_t line, const std::string& p, const std::string& v);
  // Source::Compute (Source.hpp:313-567), Cartesian directions only.
  std::array<double, 3> compute(double x, double y, double z, double t) const;
};

struct Output {  // Output.hpp:37-52
  std::string mode = "none", name = "simulation";
  double period = 0, nextprint = 1e-15, delay = 0;
  double xstart = 0, ystart = 0, zstart = 0, xstep = 0, ystep = 0, zstep = 0, xstop = 0, ystop = 0,
         zstop = 0;
  int ref_sys = 0;
  std::vector<std::array<double, 3>> probes;
  void set(uint32_t line, const std::string& p, const std::string& v);
  void initialize() { nextprint = delay; }
  bool allow_print(double t) {  // Output.hpp:300-310
    if (t >= nextprint) {
      nextprint += period;
      return true;
    }
    return false;
  }
};

struct Simulation {  // Simulation.hpp:37-50
  double duration = 0, courant = 1, step = 0, tol = 1e-8;
  std::string method = "dga", solver = "none", analytic = "false";
  bool debug = false;
  std::vector<uint32_t> sources{1};
  uint32_t mesh = 1, output = 0;
  void set(uint32_t line, const std::string& p, const std::string& v);
};

struct Mesh {  // Mesh.hpp:37-46
  std::string file = "none", name = "none", type = "none", mesher = "none";
  double scale = 1, xmin = 0, ymin = 0, zmin = 0, xmax = 0, ymax = 0, zmax = 0, xstep = 0, ystep = 0,
         zstep = 0;
  void set(uint32_t line, const std::string& p, const std::string& v);
};

struct Solid {  // Solid.hpp:37-45
  std::string type = "none";
  uint32_t material = 0;
  double sqr = 0;
  std::array<double, 3> center{0, 0, 0}, corner{0, 0, 0}, size{0, 0, 0};
  void set(uint32_t line, const std::string& p, const std::string& v);
  bool rule(double x, double y, double z) const;  // Solid.hpp:264-317
};

struct Script {
  std::map<uint32_t, Material> materials;
  std::map<uint32_t, BoundaryCondition> bcs;
  std::map<uint32_t, Mesh> meshes;
  std::map<uint32_t, Source> sources;
  std::map<uint32_t, Simulation> simulations;
  std::map<uint32_t, Output> outputs;
  std::vector<uint32_t> bnd_to_bc = std::vector<uint32_t>(100, 0);
  std::string base_dir;  // directory of the script, for relative mesh paths
  void parse(const std::string& path);
};

std::map<uint32_t, Solid> read_solids(const std::string& path);
std::string resolve_path(const std::string& base_dir, const std::string& file);

}  // namespace tf
