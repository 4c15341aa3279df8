// ORACLE — test infrastructure only (see script.hpp). Restates the reference's
// script and solids-file semantics; every setter cites the reference lines it
// follows.
#include "script.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <unistd.h>

namespace orc {

namespace msg {  // Utilities.hpp:278-317
const char* bc_unknown_type = "Unrecognized boundary condition type! Available: pec, pmc, pml";
const char* bc_unknown_parameter = "Unrecognized boundary condition parameter! Available: type";
const char* bc_unknown_direction = "Unrecognized direction! Available: +-x, +-y, +-z, r, +-t, rho";
const char* src_unknown_direction = "Unrecognized direction! Available: x, y, z";
const char* src_unknown_type =
    "Unrecognized source type!Available: e (electric field), b (magnetic field), j (current density)";
const char* src_unknown_profile = "Unrecognized source profile! Available: const, wave, gaussian";
const char* src_unknown_carrier = "Unrecognized source carrier! Available: dc, sin, cos, gaussian, ricker";
const char* coordinates_syntax = "coordinates must be inside braces {...,..,..}";
const char* unbalanced_bracket = "unbalanced bracket";
const char* too_many_coords = "Maximum of three coordinates!";
const char* too_few_coords = "Undefined end to list of coordinates!";
const char* src_unknown_bf = "Unrecognized base function! Available: sin, cos";
const char* src_unknown_parameter = "unrecognized parameter for source!";
const char* material_unknown_parameter = "Unrecognized material parameter! Available: epsilon, mu, sigma, chi";
const char* mesh_unknown_type = "Undefined mesh type! Available: tetrahedral, cartesian";
const char* mesh_inexistent_file = "Mesh input file does not exist or it is not in specified path";
const char* mesh_unknown_mesher = "Undefined mesher! Available: netgen, gmsh";
const char* mesh_unknown_parameter = "Undefined mesh parameter! Available: file, name, type, mesher, scalefactor";
const char* sim_unknown_output = "Undefined output mode type! Available: silo, probepoint, maxerror, l2norm";
const char* sim_unknown_method = "Undefined simulation method! Available: fdtd, dga, fem";
const char* sim_unknown_solver = "Unavailable solver! Available: cg, agmg";
const char* sim_unknown_parameter = "Undefined simulation parameter! Available: source, mesh, duration, output";
const char* out_unknown_parameter = "Undefined output parameter! Available: mode, period, probe, name";
const char* sim_invalid_coord_system = "Invalid system of coordinates! Available: cartesian, cylindrical, spherical";
const char* set_wo_define = "define something before setting variables";
const char* unknown_define =
    "can only define one of the following: material, mesh, refinement, boundary condition, simulation, output, "
    "source";
const char* grid_unknown_define = "Unknown primivite: can only define solid inside cartesian meshes";
const char* end_wo_define = "ending unopened definition";
const char* unknown_instruction = "Unknown instruction inside define block";
const char* unexpected_end = "File ended unexpectedly before ending definition";
const char* solid_unknown_parameter = "Unrecognized solid parameter! Available: type, radius, center, corner, size";
const char* solid_unknown_type = "Unavailable solid type! Available: sphere, box, cylinder";
const char* solid_negative_value = "Positive definite quantity forced to negative value!";
}  // namespace msg

void my_throw(uint32_t line, const std::string& m) {
  throw ScriptError("Input file error at line " + std::to_string(line) + ": " + m);
}

static bool in(const std::vector<std::string>& v, const std::string& s) {
  return std::find(v.begin(), v.end(), s) != v.end();
}

// Utilities.hpp:262-276 (allowed keyword lists).
static const std::vector<std::string> kDefinables = {"material", "source", "mesh",   "bc",
                                                     "simulation", "geometry", "output", "refinement"};
static const std::vector<std::string> kSolidTypes = {"sphere", "box", "cylinder"};
static const std::vector<std::string> kSourceTypes = {"e", "b", "j", "h", "d"};
static const std::vector<std::string> kProfiles = {"wave", "gaussian", "const"};
static const std::vector<std::string> kCarriers = {"sin", "cos", "gaussian", "dc", "ricker"};
static const std::vector<std::string> kDirections = {"x", "y", "z", "r", "psi", "rho", "phi", "theta"};
static const std::vector<std::string> kBcDirections = {"+x", "+y", "+z", "r", "+t", "rho", "-t", "-x", "-y", "-z"};
static const std::vector<std::string> kModes = {"sin", "cos"};
static const std::vector<std::string> kMeshTypes = {"tetrahedral", "cartesian", "none"};
static const std::vector<std::string> kMeshers = {"netgen", "gmsh", "none"};
static const std::vector<std::string> kOutputModes = {"silo", "probepoint", "maxerror", "l2norm"};
static const std::vector<std::string> kMethods = {"fdtd", "dga", "fem", "dgao2", "frac", "gfdtd", "fraco2", "fdtdo2"};
static const std::vector<std::string> kSolvers = {"cg", "agmg"};

// The brace-list walker shared by every `{a,b,c}` setter in the reference
// (e.g. Source.hpp:91-133): at most three entries, `,` separated, `}` closed.
static void brace_list(uint32_t line, const std::string& v, bool strip_spaces,
                       const std::function<void(int, const std::string&)>& put) {
  size_t i = 0;
  if (v.empty() || v[0] != '{') my_throw(line, msg::coordinates_syntax);
  int k = 0;
  i++;
  while (i < v.size() && v[i] != ',' && v[i] != '}') {
    std::string coord;
    while (i < v.size() && v[i] != ',' && v[i] != '}') {
      if (!(strip_spaces && v[i] == ' ')) coord.push_back(v[i]);
      i++;
    }
    if (i == v.size()) my_throw(line, msg::unbalanced_bracket);
    if (k < 3) {
      put(k, coord);
      k++;
    } else {
      my_throw(line, msg::too_many_coords);
    }
    if (v[i] == ',') i++;
  }
  if (i == v.size()) my_throw(line, msg::too_few_coords);
}

void Material::set(uint32_t line, const std::string& p, const std::string& v) {
  // Material.hpp:45-316
  auto sym = [&](Mat3& m, int a, int b) { m.m[a][b] = m.m[b][a] = std::stod(v); };
  if (p == "epsilon") eps = Mat3::diag(EPS0 * std::stod(v));
  else if (p == "epsilon_xy") sym(eps, 0, 1);
  else if (p == "epsilon_xz") sym(eps, 0, 2);
  else if (p == "epsilon_yz") sym(eps, 1, 2);
  else if (p == "mu") mu = Mat3::diag(MU0 * std::stod(v));
  else if (p == "mu_xy") sym(mu, 0, 1);
  else if (p == "mu_xz") sym(mu, 0, 2);
  else if (p == "mu_yz") sym(mu, 1, 2);
  else if (p == "sigma") sigma = Mat3::diag(std::stod(v));
  else if (p == "sigma_xy") sym(sigma, 0, 1);
  else if (p == "sigma_xz") sym(sigma, 0, 2);
  else if (p == "sigma_yz") sym(sigma, 1, 2);
  else if (p == "chi") chi = Mat3::diag(std::stod(v));
  else if (p == "chi_xy") sym(chi, 0, 1);
  else if (p == "chi_xz") sym(chi, 0, 2);
  else if (p == "chi_yz") sym(chi, 1, 2);
  else if (p == "eps_vec") brace_list(line, v, false, [&](int k, const std::string& c) { eps.m[k][k] = EPS0 * std::stod(c); });
  else if (p == "mu_vec") brace_list(line, v, false, [&](int k, const std::string& c) { mu.m[k][k] = MU0 * std::stod(c); });
  else if (p == "sigma_vec") brace_list(line, v, false, [&](int k, const std::string& c) { sigma.m[k][k] = std::stod(c); });
  else if (p == "chi_vec") brace_list(line, v, false, [&](int k, const std::string& c) { chi.m[k][k] = std::stod(c); });
  else my_throw(line, msg::material_unknown_parameter);
}

void BoundaryCondition::set(uint32_t line, const std::string& p, const std::string& v) {
  // BoundaryCondition.hpp:45-125
  if (p == "type") {
    if (v == "pml") type = v;
    else if (v == "pmc" || v == "pec") { type = v; val = 0; }
    else my_throw(line, msg::bc_unknown_type);
  } else if (p == "direction") {
    if (!in(kBcDirections, v)) my_throw(line, msg::bc_unknown_direction);
    dir = v;
  } else if (p == "width") width = std::stod(v);
  else if (p == "surface") surfs.push_back(std::stoi(v));
  else if (p == "surfaces") {
    size_t i = 0;
    if (v.empty() || v[0] != '{') my_throw(line, msg::coordinates_syntax);
    i++;
    while (i < v.size() && v[i] != '}') {
      std::string c;
      while (i < v.size() && v[i] != ',' && v[i] != '}') c.push_back(v[i++]);
      if (i == v.size()) my_throw(line, msg::unbalanced_bracket);
      surfs.push_back(std::stoi(c));
      if (v[i] == ',') i++;
    }
    if (i == v.size()) my_throw(line, msg::unbalanced_bracket);
  } else my_throw(line, msg::bc_unknown_parameter);
}

void Source::set(uint32_t line, const std::string& p, const std::string& v) {
  // Source.hpp:60-300
  if (p == "direction") {
    if (!in(kDirections, v)) my_throw(line, msg::src_unknown_direction);
    dir = v;
  } else if (p == "type") {
    if (!in(kSourceTypes, v)) my_throw(line, msg::src_unknown_type);
    st = v;
  } else if (p == "profile") {
    if (!in(kProfiles, v)) my_throw(line, msg::src_unknown_profile);
    prof = v;
  } else if (p == "carrier") {
    if (!in(kCarriers, v)) my_throw(line, msg::src_unknown_carrier);
    carrier = v;
  } else if (p == "center") brace_list(line, v, false, [&](int k, const std::string& c) { center[k] = std::stod(c); });
  else if (p == "wavevector") brace_list(line, v, false, [&](int k, const std::string& c) { kvec[k] = std::stod(c); });
  else if (p == "location") brace_list(line, v, false, [&](int k, const std::string& c) { location[k] = std::stod(c); });
  else if (p == "mode") brace_list(line, v, true, [&](int k, const std::string& c) { bfuncs[k] = c; });
  else if (p == "Xmode" || p == "Ymode" || p == "Zmode") {
    if (!in(kModes, v)) my_throw(line, msg::src_unknown_bf);
    bfuncs[p[0] - 'X'] = v;
  } else if (p == "amplitude") amp = std::stod(v);
  else if (p == "delay") delay = std::stod(v);
  else if (p == "impedance") impedance = std::stod(v);
  else if (p == "frequency") freq = std::stod(v);
  else if (p == "radius") radius = std::stod(v);
  else if (p == "decay") decay = std::stod(v);
  else if (p == "width") width = std::stod(v);
  else if (p == "kx") kvec[0] = std::stod(v);
  else if (p == "ky") kvec[1] = std::stod(v);
  else if (p == "kz") kvec[2] = std::stod(v);
  else if (p == "surface") surfaces.push_back(std::stoi(v));
  else my_throw(line, msg::src_unknown_parameter);
}

std::array<double, 3> Source::compute(double x, double y, double z, double t) const {
  // Source.hpp:313-325 (carrier) and :525-565 (Cartesian spatial profile).
  // The reference forms the phase 2*PI*f*(t-delay) with a long double PI.
  double ret = amp;
  if (st == "j") ret *= impedance;
  if (carrier == "sin") ret *= std::sin((double)(2 * PI_L * freq * (t - delay)));
  else if (carrier == "cos") ret *= amp * std::cos((double)(2 * PI_L * freq * (t - delay)));
  else if (carrier == "gaussian") ret *= std::exp(-std::pow(t - delay, 2) / std::pow(width, 2));
  else if (carrier == "ricker") {
    double a = (double)(PI_L * freq * (t - delay));
    ret *= (1 - 2 * std::pow(a, 2)) * std::exp(-std::pow(a, 2));
  }
  const double p[3] = {x, y, z};
  if (decay != 0)
    ret *= std::pow(std::pow(p[0] - center[0], 2) + std::pow(p[1] - center[1], 2) + std::pow(p[2] - center[2], 2),
                    -0.5 * decay);
  if (prof == "gaussian") {
    double e = -((std::pow(p[0] - center[0], 2) + std::pow(p[1] - center[1], 2) + std::pow(p[2] - center[2], 2)) /
                 std::pow(radius, 2));
    ret *= std::exp(e);
  } else if (prof == "wave") {
    for (int j = 0; j < 3; j++) {
      if (bfuncs[j] == "sin") ret *= std::sin((double)(2 * PI_L * kvec[j] * (p[j] - center[j])));
      else if (bfuncs[j] == "cos") ret *= std::cos((double)(2 * PI_L * kvec[j] * (p[j] - center[j])));
    }
  }
  if (dir == "x") return {ret, 0, 0};
  if (dir == "y") return {0, ret, 0};
  return {0, 0, ret};
}

void Output::set(uint32_t line, const std::string& p, const std::string& v) {
  // Output.hpp:58-298.  Probe and grid coordinates go through std::stof.
  if (p == "mode") {
    if (!in(kOutputModes, v)) my_throw(line, msg::sim_unknown_output);
    mode = v;
  } else if (p == "radiator") {
    (void)std::stof(v);
  } else if (p == "delay") nextprint = delay = std::stod(v);
  else if (p == "coordinates") {
    if (v == "cartesian") ref_sys = 0;
    else if (v == "cylindrical") ref_sys = 1;
    else if (v == "spherical") ref_sys = 2;
    else my_throw(line, msg::sim_invalid_coord_system);
  } else if (p == "probe") {
    std::array<double, 3> pp{0, 0, 0};
    brace_list(line, v, false, [&](int k, const std::string& c) { pp[k] = std::stof(c); });
    probes.push_back(pp);
  } else if (p == "period") period = std::stof(v);
  else if (p == "xgrid" || p == "ygrid" || p == "zgrid") {
    double *st, *sp, *so;
    if (p[0] == 'x') { st = &xstart; sp = &xstep; so = &xstop; }
    else if (p[0] == 'y') { st = &ystart; sp = &ystep; so = &ystop; }
    else { st = &zstart; sp = &zstep; so = &zstop; }
    brace_list(line, v, false, [&](int k, const std::string& c) {
      double d = std::stof(c);
      if (k == 0) *st = d;
      else if (k == 1) *sp = d;
      else *so = d;
    });
  } else if (p == "grid") {
    if (v == "on") {
      for (double z = zstart; z <= zstop; z += zstep)
        for (double y = ystart; y <= ystop; y += ystep)
          for (double x = xstart; x <= xstop; x += xstep) probes.push_back({x, y, z});
    } else if (v != "off") my_throw(line, msg::out_unknown_parameter);
  } else if (p == "error") {
    if (v != "on" && v != "off") my_throw(line, msg::out_unknown_parameter);
  } else if (p == "name") name = v;
  else my_throw(line, msg::out_unknown_parameter);
}

void Simulation::set(uint32_t line, const std::string& p, const std::string& v) {
  // Simulation.hpp:52-97
  if (p == "source") {
    sources.push_back((uint32_t)std::stod(v));
    std::sort(sources.begin(), sources.end());
    sources.erase(std::unique(sources.begin(), sources.end()), sources.end());
  } else if (p == "mesh") mesh = (uint32_t)std::stod(v);
  else if (p == "duration") duration = std::stod(v);
  else if (p == "courant") courant = std::stod(v);
  else if (p == "step") step = std::stod(v);
  else if (p == "output") output = (uint32_t)std::stod(v);
  else if (p == "method") {
    if (!in(kMethods, v)) my_throw(line, msg::sim_unknown_method);
    method = v;
  } else if (p == "solver") {
    if (!in(kSolvers, v)) my_throw(line, msg::sim_unknown_solver);
    solver = v;
  } else if (p == "tolerance") tol = std::stod(v);
  else if (p == "analytic") analytic = v;
  else if (p == "debug") {
    if (v == "true") debug = true;
    else if (v == "false") debug = false;
    else my_throw(line, msg::sim_unknown_parameter);
  } else my_throw(line, msg::sim_unknown_parameter);
}

static bool file_exists(const std::string& f) {
  std::ifstream t(f.c_str());
  return t.is_open();
}

std::string resolve_path(const std::string& base_dir, const std::string& file) {
  if (file_exists(file) || file.empty() || file[0] == '/' || base_dir.empty()) return file;
  std::string alt = base_dir + "/" + file;
  return file_exists(alt) ? alt : file;
}

void Mesh::set(uint32_t line, const std::string& p, const std::string& v) {
  // Mesh.hpp:44-251
  if (p == "file") {
    if (!file_exists(v)) my_throw(line, msg::mesh_inexistent_file);
    file = v;
  } else if (p == "name") name = v;
  else if (p == "type") {
    if (!in(kMeshTypes, v)) my_throw(line, msg::mesh_unknown_type);
    type = v;
  } else if (p == "mesher") {
    if (!in(kMeshers, v)) my_throw(line, msg::mesh_unknown_mesher);
    mesher = v;
  } else if (p == "xgrid" || p == "ygrid" || p == "zgrid") {
    double *mn, *st, *mx;
    if (p[0] == 'x') { mn = &xmin; st = &xstep; mx = &xmax; }
    else if (p[0] == 'y') { mn = &ymin; st = &ystep; mx = &ymax; }
    else { mn = &zmin; st = &zstep; mx = &zmax; }
    brace_list(line, v, false, [&](int k, const std::string& c) {
      double d = std::stod(c);
      if (k == 0) *mn = d;
      else if (k == 1) *st = d;
      else *mx = d;
    });
  } else if (p == "scalefactor") scale = std::stod(v);
  else my_throw(line, msg::mesh_unknown_parameter);
}

void Solid::set(uint32_t line, const std::string& p, const std::string& v) {
  // Solid.hpp:47-262
  if (p == "type") {
    if (!in(kSolidTypes, v)) my_throw(line, msg::solid_unknown_type);
    type = v;
  } else if (p == "material") material = (uint32_t)std::atoi(v.c_str());
  else if (p == "radius") {
    double r = std::stod(v);
    if (r <= 0) my_throw(line, msg::solid_negative_value);
    sqr = std::pow(r, 2);
  } else if (p == "center") brace_list(line, v, false, [&](int k, const std::string& c) { center[k] = std::stod(c); });
  else if (p == "corner") brace_list(line, v, false, [&](int k, const std::string& c) { corner[k] = std::stod(c); });
  else if (p == "size") brace_list(line, v, false, [&](int k, const std::string& c) {
    size[k] = std::stod(c);
    if (size[k] < 0) my_throw(line, msg::solid_negative_value);
  });
  else my_throw(line, msg::solid_unknown_parameter);
}

bool Solid::rule(double x, double y, double z) const {
  // Solid.hpp:264-317
  if (type == "sphere") {
    double d0 = x - center[0], d1 = y - center[1], d2 = z - center[2];
    return d0 * d0 + d1 * d1 + d2 * d2 <= sqr;
  }
  if (type == "box") {
    double d[3] = {x - corner[0], y - corner[1], z - corner[2]};
    for (int k = 0; k < 3; k++)
      if (d[k] > size[k] || d[k] < 0) return false;
    return true;
  }
  if (type == "cylinder") {
    double sn2 = size[0] * size[0] + size[1] * size[1] + size[2] * size[2];
    if (std::sqrt(sn2) == 0) return false;
    double pd[3] = {x - center[0], y - center[1], z - center[2]};
    double dot = pd[0] * size[0] + pd[1] * size[1] + pd[2] * size[2];
    if (dot < -1e-12 || dot > (sn2 + 1e-12)) return false;
    double dsq = (pd[0] * pd[0] + pd[1] * pd[1] + pd[2] * pd[2]) - dot * dot / sn2;
    return !(dsq > (sqr + 1e-12));
  }
  return false;
}

// Line splitter shared by the script and solids readers: `%s %s %s` tokens that
// persist across lines (the reference keeps its char buffers outside the loop),
// and a brace value re-joined from the raw line (Discretization.hpp:144-161).
struct LineState {
  char action[256] = {0}, token[256] = {0}, value[256] = {0};
};

static bool split_line(const std::string& line, LineState& s, std::string& instr, std::string& tok,
                       std::string& val, uint32_t ln, bool for_set) {
  const char* c = line.c_str();
  if (line.empty() || c[0] == '#' || c[0] == '\n') return false;
  std::sscanf(c, "%255s %255s %255s", s.action, s.token, s.value);
  instr = s.action;
  tok = s.token;
  val = s.value;
  if (instr.empty() || instr[0] == '#') return false;
  (void)ln;
  (void)for_set;
  return true;
}

static void rejoin_brace(const std::string& line, const LineState& s, std::string& val, uint32_t ln) {
  if (s.value[0] != '{') return;
  size_t i = line.find('{');
  val.clear();
  while (i < line.size() && line[i] != '}') val.push_back(line[i++]);
  if (i == line.size()) my_throw(ln, msg::unbalanced_bracket);
  val.push_back('}');
}

void Script::parse(const std::string& path) {
  // Discretization.hpp:45-211
  std::ifstream f(path.c_str());
  if (!f.is_open()) throw ScriptError("cannot open script file: " + path);
  size_t slash = path.rfind('/');
  base_dir = slash == std::string::npos ? std::string() : path.substr(0, slash);
  std::string line, instr, tok, val, thing;
  LineState s;
  bool in_def = false;
  uint32_t label = 0, ln = 1;
  std::string cwd_saved;
  while (std::getline(f, line)) {
    if (split_line(line, s, instr, tok, val, ln, true)) {
      if (!in_def) {
        if (instr != "DEFINE") my_throw(ln, msg::set_wo_define);
        if (!in(kDefinables, tok)) my_throw(ln, msg::unknown_define);
        thing = tok;
        label = (uint32_t)std::stoi(val);
        in_def = true;
        if (thing == "material") materials[label] = Material();
        else if (thing == "bc") bcs[label] = BoundaryCondition();
        else if (thing == "mesh") meshes[label] = Mesh();
        else if (thing == "source") sources[label] = Source();
        else if (thing == "simulation") simulations[label] = Simulation();
        else if (thing == "output") outputs[label] = Output();
      } else if (instr == "END") {
        if (tok != thing || (uint32_t)std::atoi(s.value) != label) my_throw(ln, msg::end_wo_define);
        in_def = false;
        if (thing == "bc")
          for (auto sf : bcs[label].surfs) {
            if (sf >= bnd_to_bc.size())
              throw ScriptError("bc surface label " + std::to_string(sf) + " outside the 100-slot label table");
            bnd_to_bc[sf] = label;
          }
      } else if (instr != "SET") {
        my_throw(ln, msg::unknown_instruction);
      } else {
        rejoin_brace(line, s, val, ln);
        if (thing == "material") materials[label].set(ln, tok, val);
        else if (thing == "bc") bcs[label].set(ln, tok, val);
        else if (thing == "mesh") {
          // Mesh.hpp:46-60 checks the file relative to the working directory;
          // a path relative to the script's own directory is also accepted.
          if (tok == "file") val = resolve_path(base_dir, val);
          meshes[label].set(ln, tok, val);
        } else if (thing == "source") sources[label].set(ln, tok, val);
        else if (thing == "simulation") simulations[label].set(ln, tok, val);
        else if (thing == "output") outputs[label].set(ln, tok, val);
        else if (thing == "refinement" || thing == "geometry")
          throw ScriptError("refinement/geometry primitives are outside the time-stepping path");
        else my_throw(ln, msg::unknown_define);
      }
    }
    ln++;
  }
  if (in_def) my_throw(ln, msg::unexpected_end);
}

std::map<uint32_t, Solid> read_solids(const std::string& path) {
  // Discretization.hpp:4219-4345
  std::map<uint32_t, Solid> solids;
  std::ifstream f(path.c_str());
  if (!f.is_open()) throw ScriptError("Invalid mesh file name");
  std::string line, instr, tok, val, thing;
  LineState s;
  bool in_def = false;
  uint32_t label = 0, ln = 1;
  static const std::vector<std::string> kMeshDefinables = {"grid", "solid"};
  const std::string pre = "In cartesian mesh definition file: ";
  auto thr = [&](const char* m) { throw ScriptError(pre + "Input file error at line " + std::to_string(ln) + ": " + m); };
  while (std::getline(f, line)) {
    if (split_line(line, s, instr, tok, val, ln, true)) {
      if (!in_def) {
        if (instr != "DEFINE") thr(msg::set_wo_define);
        if (!in(kMeshDefinables, tok)) thr(msg::grid_unknown_define);
        thing = tok;
        label = (uint32_t)std::stod(val);
        in_def = true;
        if (thing == "solid") solids[label] = Solid();
      } else if (instr == "END") {
        if (tok != thing || (uint32_t)std::atoi(s.value) != label) thr(msg::end_wo_define);
        in_def = false;
      } else if (instr != "SET") {
        thr(msg::unknown_instruction);
      } else {
        rejoin_brace(line, s, val, ln);
        if (thing == "solid") solids[label].set(ln, tok, val);
        else thr(msg::grid_unknown_define);
      }
    }
    ln++;
  }
  if (in_def) thr(msg::unexpected_end);
  return solids;
}

}  // namespace orc
