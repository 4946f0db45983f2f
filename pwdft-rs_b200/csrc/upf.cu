// UPF v2 norm-conserving pseudopotential reader behind the C-ABI (host code
// only): the parse of parse_upf_body (pseudopotential/upf/parse.rs:20-135)
// with the attribute and data-block scanning of upf/xml.rs. Fields are found
// by their first textual occurrence, as the reference does, and converted to
// the units pwgpu_system's radial fields take: r, rab in Å; V_loc in eV;
// r·β(r) divided by sqrt(Å per bohr); D_ij in eV; PP_RHOATOM per Å; the NLCC
// core charge in e/Å^3. A caller without Python (the reference's Rust host,
// a serving front end) reads a species once and fills the radial part of
// pwgpu_system from it.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "handle.hpp"
#include "../../include/pwgpu.h"

struct pwgpu_upf {
  std::string element;
  double z_valence = 0.0;
  int l_max = 0;
  int mesh = 0;
  std::vector<double> r, rab, v_local, dij, rho_atom, core;
  std::vector<std::vector<double>> beta;
  std::vector<int> beta_l;
};

namespace {

using pwgpu::fail;

constexpr double kBohrToAng = 0.529177210903;
constexpr double kRyToEv = 13.605693122994;
constexpr double kBohr3ToAng3 = kBohrToAng * kBohrToAng * kBohrToAng;

struct ParseError {
  std::string msg;
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// the value of the first name="..." in text, or false
bool attr(const std::string& text, const std::string& name, std::string& out) {
  const std::string pat = name + "=\"";
  size_t s = text.find(pat);
  if (s == std::string::npos) return false;
  s += pat.size();
  const size_t e = text.find('"', s);
  if (e == std::string::npos) return false;
  out = text.substr(s, e - s);
  return true;
}

// a whole token as a double (every character consumed)
bool to_double(const std::string& tok, double& v) {
  if (tok.empty()) return false;
  errno = 0;
  char* end = nullptr;
  v = std::strtod(tok.c_str(), &end);
  // strtod also reads hexadecimal floats, which the reference's parser does not
  return end == tok.c_str() + tok.size() && tok.find_first_of("xX") == std::string::npos;
}

bool to_int(const std::string& tok, int& v) {
  if (tok.empty()) return false;
  errno = 0;
  char* end = nullptr;
  const long x = std::strtol(tok.c_str(), &end, 10);
  if (end != tok.c_str() + tok.size() || errno == ERANGE || x < INT32_MIN || x > INT32_MAX) return false;
  v = (int)x;
  return true;
}

template <typename T, typename F>
T header_number(const std::string& text, const char* name, F conv) {
  std::string s;
  if (!attr(text, name, s)) throw ParseError{std::string("missing ") + name};
  T v{};
  if (!conv(trim(s), v)) throw ParseError{std::string(name) + " parse error: '" + trim(s) + "'"};
  return v;
}

// the whitespace-separated numbers between <tag ...> and </tag>, which must
// number exactly `expected`
std::vector<double> block(const std::string& text, const std::string& tag, long expected) {
  const size_t p = text.find("<" + tag);
  if (p == std::string::npos) throw ParseError{"missing tag <" + tag + ">"};
  const size_t gt = text.find('>', p);
  if (gt == std::string::npos) throw ParseError{"malformed tag <" + tag + ">"};
  const size_t end = text.find("</" + tag + ">", gt + 1);
  if (end == std::string::npos) throw ParseError{"missing closing tag </" + tag + ">"};
  std::vector<double> vals;
  size_t i = gt + 1;
  while (i < end) {
    while (i < end && std::isspace((unsigned char)text[i])) ++i;
    size_t j = i;
    while (j < end && !std::isspace((unsigned char)text[j])) ++j;
    if (j > i) {
      double v;
      const std::string tok = text.substr(i, j - i);
      if (!to_double(tok, v)) throw ParseError{"float parse error in " + tag + ": '" + tok + "'"};
      vals.push_back(v);
    }
    i = j;
  }
  if ((long)vals.size() != expected)
    throw ParseError{tag + ": expected " + std::to_string(expected) + " values, got " + std::to_string(vals.size())};
  return vals;
}

int beta_l(const std::string& text, const std::string& tag) {
  const size_t p = text.find("<" + tag);
  if (p == std::string::npos) throw ParseError{"missing tag <" + tag + ">"};
  const size_t gt = text.find('>', p);
  if (gt == std::string::npos) throw ParseError{"malformed tag <" + tag + ">"};
  std::string s;
  if (!attr(text.substr(p, gt - p), "angular_momentum", s))
    throw ParseError{"missing angular_momentum attribute in " + tag};
  int l;
  if (!to_int(trim(s), l)) throw ParseError{tag + ": angular_momentum parse error"};
  if (l < 0) throw ParseError{tag + ": angular_momentum must be non-negative (got " + std::to_string(l) + ")"};
  return l;
}

void scale(std::vector<double>& v, double f, bool divide) {
  for (double& x : v) x = divide ? x / f : x * f;
}

pwgpu_upf* parse(const std::string& text) {
  if (text.find("<UPF") == std::string::npos && text.find("<PP_HEADER") == std::string::npos)
    throw ParseError{"unrecognized pseudopotential format (only UPF v2 is supported)"};
  std::string el;
  if (!attr(text, "element", el)) throw ParseError{"missing element in PP_HEADER"};
  auto* u = new pwgpu_upf();
  try {
    u->element = trim(el);
    u->z_valence = header_number<double>(text, "z_valence", to_double);
    u->l_max = header_number<int>(text, "l_max", to_int);
    const int nproj = header_number<int>(text, "number_of_proj", to_int);
    u->mesh = header_number<int>(text, "mesh_size", to_int);
    if (nproj < 0 || u->mesh < 0) throw ParseError{"negative number_of_proj or mesh_size"};
    u->r = block(text, "PP_R", u->mesh);
    scale(u->r, kBohrToAng, false);
    u->rab = block(text, "PP_RAB", u->mesh);
    scale(u->rab, kBohrToAng, false);
    u->v_local = block(text, "PP_LOCAL", u->mesh);
    scale(u->v_local, kRyToEv, false);
    const double sq = std::sqrt(kBohrToAng);
    for (int i = 1; i <= nproj; ++i) {
      const std::string tag = "PP_BETA." + std::to_string(i);
      u->beta_l.push_back(beta_l(text, tag));
      u->beta.push_back(block(text, tag, u->mesh));
      scale(u->beta.back(), sq, true);
    }
    u->dij = block(text, "PP_DIJ", (long)nproj * nproj);
    scale(u->dij, kRyToEv, false);
    try {
      u->rho_atom = block(text, "PP_RHOATOM", u->mesh);
      scale(u->rho_atom, kBohrToAng, true);
    } catch (const ParseError&) {
      u->rho_atom.assign(u->mesh, 0.0);
    }
    const bool nlcc = text.find("core_correction=\"T\"") != std::string::npos ||
                      text.find("core_correction=\"t\"") != std::string::npos ||
                      text.find("nlcc=.true.") != std::string::npos;
    if (nlcc) {
      try {
        u->core = block(text, "PP_NLCC", u->mesh);
        scale(u->core, kBohr3ToAng3, true);
      } catch (const ParseError&) {
        u->core.assign(u->mesh, 0.0);
      }
    }
  } catch (...) {
    delete u;
    throw;
  }
  return u;
}

}  // namespace

extern "C" {

pwgpu_status pwgpu_upf_parse(const char* text, int64_t len, pwgpu_upf** out) {
  if (!text || !out || len < 0) return fail(PWGPU_E_INVALID, "pwgpu_upf_parse: NULL argument or negative length");
  *out = nullptr;
  try {
    *out = parse(std::string(text, (size_t)len));
  } catch (const ParseError& e) {
    return fail(PWGPU_E_PARSE, "UPF: " + e.msg);
  } catch (const std::bad_alloc&) {
    return fail(PWGPU_E_OOM, "pwgpu_upf_parse: out of host memory");
  }
  return PWGPU_OK;
}

pwgpu_status pwgpu_upf_load(const char* path, pwgpu_upf** out) {
  if (!path || !out) return fail(PWGPU_E_INVALID, "pwgpu_upf_load: NULL argument");
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(PWGPU_E_INVALID, std::string("pwgpu_upf_load: cannot open ") + path);
  std::string text;
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  const bool bad = std::ferror(f) != 0;
  std::fclose(f);
  if (bad) return fail(PWGPU_E_INVALID, std::string("pwgpu_upf_load: read error on ") + path);
  return pwgpu_upf_parse(text.data(), (int64_t)text.size(), out);
}

pwgpu_status pwgpu_upf_get_info(const pwgpu_upf* u, pwgpu_upf_info* info) {
  if (!u || !info) return fail(PWGPU_E_INVALID, "pwgpu_upf_get_info: NULL argument");
  std::memset(info, 0, sizeof(*info));
  std::snprintf(info->element, sizeof(info->element), "%s", u->element.c_str());
  info->z_valence = u->z_valence;
  info->l_max = u->l_max;
  info->n_proj = (int32_t)u->beta.size();
  info->mesh = u->mesh;
  info->has_nlcc = u->core.empty() ? 0 : 1;
  int any = 0;
  for (double x : u->rho_atom) any |= std::fabs(x) > 1e-20;
  info->has_rho_atom = any;
  return PWGPU_OK;
}

pwgpu_status pwgpu_upf_get_array(const pwgpu_upf* u, int32_t which, int32_t index, double* out, int64_t capacity) {
  if (!u || !out) return fail(PWGPU_E_INVALID, "pwgpu_upf_get_array: NULL argument");
  const std::vector<double>* v = nullptr;
  switch (which) {
    case PWGPU_UPF_R: v = &u->r; break;
    case PWGPU_UPF_RAB: v = &u->rab; break;
    case PWGPU_UPF_LOCAL: v = &u->v_local; break;
    case PWGPU_UPF_BETA:
      if (index < 0 || index >= (int32_t)u->beta.size())
        return fail(PWGPU_E_INVALID, "pwgpu_upf_get_array: projector index out of range");
      v = &u->beta[index];
      break;
    case PWGPU_UPF_DIJ: v = &u->dij; break;
    case PWGPU_UPF_RHOATOM: v = &u->rho_atom; break;
    case PWGPU_UPF_NLCC: v = &u->core; break;
    default: return fail(PWGPU_E_INVALID, "pwgpu_upf_get_array: unknown array");
  }
  if (capacity < (int64_t)v->size())
    return fail(PWGPU_E_INVALID, "pwgpu_upf_get_array: output holds " + std::to_string(capacity) + " values, need " +
                                     std::to_string(v->size()));
  if (!v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return PWGPU_OK;
}

pwgpu_status pwgpu_upf_get_beta_l(const pwgpu_upf* u, int32_t* l) {
  if (!u || !l) return fail(PWGPU_E_INVALID, "pwgpu_upf_get_beta_l: NULL argument");
  for (size_t i = 0; i < u->beta_l.size(); ++i) l[i] = u->beta_l[i];
  return PWGPU_OK;
}

pwgpu_status pwgpu_upf_free(pwgpu_upf* u) {
  delete u;
  return PWGPU_OK;
}

}  // extern "C"
