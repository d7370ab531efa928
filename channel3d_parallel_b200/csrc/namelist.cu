// Reader of the reference's &params namelist (src/input_output.f90:21-132):
// same variable list (:27-40), same defaults (:43-62), case-insensitive keys,
// '!' comments, Fortran d/e exponents, logicals and quoted strings.
#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <string>

#include "c3d_internal.cuh"

namespace c3d {

static std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

static bool to_double(const std::string& tok, double& v) {
  std::string t = tok;
  for (auto& c : t) if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return end && *end == '\0' && !t.empty();
}

static bool to_int(const std::string& tok, int& v) {
  char* end = nullptr;
  long r = std::strtol(tok.c_str(), &end, 10);
  if (!end || *end != '\0' || tok.empty()) return false;
  v = (int)r;
  return true;
}

int parse_namelist(const std::string& text, Params& p, std::string& err) {
  // strip comments outside quotes
  std::string body;
  {
    char q = 0;
    for (size_t i = 0; i < text.size(); ++i) {
      char c = text[i];
      if (q) { body += c; if (c == q) q = 0; continue; }
      if (c == '\'' || c == '"') { q = c; body += c; continue; }
      if (c == '!') { while (i < text.size() && text[i] != '\n') ++i; body += '\n'; continue; }
      body += c;
    }
  }
  std::string lb = lower(body);
  size_t g = lb.find("&params");
  if (g == std::string::npos) { err = "no &params group found"; return C3D_ERR_PARAM; }
  size_t pos = g + 7;
  // the group ends at a '/' outside quotes
  size_t end = std::string::npos;
  {
    char q = 0;
    for (size_t i = pos; i < body.size(); ++i) {
      char c = body[i];
      if (q) { if (c == q) q = 0; continue; }
      if (c == '\'' || c == '"') { q = c; continue; }
      if (c == '/') { end = i; break; }
    }
  }
  if (end == std::string::npos) { err = "&params group is not terminated by '/'"; return C3D_ERR_PARAM; }
  std::string grp = body.substr(pos, end - pos);
  // split into key = value items separated by newlines or commas
  size_t i = 0;
  while (i < grp.size()) {
    while (i < grp.size() && (std::isspace((unsigned char)grp[i]) || grp[i] == ',')) ++i;
    if (i >= grp.size()) break;
    size_t eq = grp.find('=', i);
    if (eq == std::string::npos) { err = "malformed namelist item near '" + trim(grp.substr(i, 20)) + "'"; return C3D_ERR_PARAM; }
    std::string key = lower(trim(grp.substr(i, eq - i)));
    size_t v0 = eq + 1;
    while (v0 < grp.size() && (grp[v0] == ' ' || grp[v0] == '\t')) ++v0;
    std::string val;
    size_t v1;
    if (v0 < grp.size() && (grp[v0] == '\'' || grp[v0] == '"')) {
      char q = grp[v0];
      v1 = grp.find(q, v0 + 1);
      if (v1 == std::string::npos) { err = "unterminated string for " + key; return C3D_ERR_PARAM; }
      val = grp.substr(v0 + 1, v1 - v0 - 1);
      ++v1;
    } else {
      v1 = v0;
      while (v1 < grp.size() && grp[v1] != '\n' && grp[v1] != ',') ++v1;
      val = trim(grp.substr(v0, v1 - v0));
    }
    i = v1;
    double dv = 0;
    int iv = 0;
    auto need_real = [&](double& dst) -> int {
      if (!to_double(val, dv)) { err = "bad real for " + key + ": '" + val + "'"; return C3D_ERR_PARAM; }
      dst = dv;
      return 0;
    };
    auto need_int = [&](int& dst) -> int {
      if (!to_int(val, iv)) { err = "bad integer for " + key + ": '" + val + "'"; return C3D_ERR_PARAM; }
      dst = iv;
      return 0;
    };
    int rc = 0;
    if (key == "lxp") rc = need_real(p.Lxp);
    else if (key == "lzp") rc = need_real(p.Lzp);
    else if (key == "ly_channel") rc = need_real(p.Ly_channel);
    else if (key == "alpha_stretch") rc = need_real(p.alpha_stretch);
    else if (key == "nx_global") rc = need_int(p.nx_global);
    else if (key == "ny_global") rc = need_int(p.ny_global);
    else if (key == "nz_global") rc = need_int(p.nz_global);
    else if (key == "nxb") rc = need_int(p.nxb);
    else if (key == "nzb") rc = need_int(p.nzb);
    else if (key == "cfl") rc = need_real(p.CFL);
    else if (key == "nu") rc = need_real(p.nu);
    else if (key == "dpdx") rc = need_real(p.dPdx);
    else if (key == "dpdz") rc = need_real(p.dPdz);
    else if (key == "qflow_x_0") rc = need_real(p.Qflow_x_0);
    else if (key == "qflow_z_0") rc = need_real(p.Qflow_z_0);
    else if (key == "x_mass_cte") rc = need_int(p.x_mass_cte);
    else if (key == "y_mass_cte") rc = need_int(p.y_mass_cte);
    else if (key == "z_mass_cte") rc = need_int(p.z_mass_cte);
    else if (key == "nsteps") rc = need_int(p.nsteps);
    else if (key == "nsave") rc = need_int(p.nsave);
    else if (key == "nstats") rc = need_int(p.nstats);
    else if (key == "nmonitor") rc = need_int(p.nmonitor);
    else if (key == "filein") p.filein = val;
    else if (key == "fileout") p.fileout = val;
    else if (key == "nstep_init") rc = need_int(p.nstep_init);
    else if (key == "t_init") rc = need_real(p.t_init);
    else if (key == "init_type") rc = need_int(p.init_type);
    else if (key == "grid_type") rc = need_int(p.grid_type);
    else if (key == "body_type") p.body_type = lower(trim(val));
    else if (key == "exterior_pressure_gradient") {
      std::string t = lower(trim(val));
      while (!t.empty() && t[0] == '.') t.erase(0, 1);
      if (!t.empty() && t[0] == 't') p.exterior_pressure_gradient = true;
      else if (!t.empty() && t[0] == 'f') p.exterior_pressure_gradient = false;
      else { err = "bad logical for " + key; rc = C3D_ERR_PARAM; }
    }
    else if (key == "body_param_1") rc = need_real(p.body_param_1);
    else if (key == "body_param_2") rc = need_real(p.body_param_2);
    else if (key == "body_param_3") rc = need_real(p.body_param_3);
    else if (key == "body_param_4") rc = need_real(p.body_param_4);   // extension
    else if (key == "body_ramp_up_time") rc = need_real(p.body_ramp_up_time);
    else if (key == "min_buffer_width") rc = need_real(p.min_buffer_width);
    else if (key == "cg_tol") rc = need_real(p.cg_tol);
    else if (key == "cg_max_iter") rc = need_int(p.cg_max_iter);
    else if (key == "perturb_scale") rc = need_real(p.perturb_scale);
    else { err = "unknown namelist variable '" + key + "'"; rc = C3D_ERR_PARAM; }
    if (rc) return rc;
  }
  return 0;
}

}  // namespace c3d
