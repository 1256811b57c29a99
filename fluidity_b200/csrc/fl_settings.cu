// fl_settings.cu -- settings-file dispatch: the reference's
// Settings::from_string / from_file (setting/settings.hpp:50-105) and the
// "simulator : { ... }" block that OptionManager::create turns into a
// SimulatorImpl type (setting/simulator_parameter.hpp:29-105,
// setting/option_manager.hpp:129-246), mapped to this library's run-time
// policy bits.  Host code only.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fluidity_b200.h"
#include "fl_internal.cuh"

namespace {

struct Setting {
  std::string name, value;
  bool complex = false;
};

void remove_chars(std::string& s, const char* chars) {
  std::string out;
  out.reserve(s.size());
  for (char c : s) {
    bool drop = false;
    for (const char* p = chars; *p; ++p) drop |= (c == *p);
    if (!drop) out.push_back(c);
  }
  s.swap(out);
}

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n'))
    --b;
  return s.substr(a, b - a);
}

// Settings::from_string: "<name> : <value>" pairs; a value runs to the next
// ',' at nesting depth 0 or to the '}' that closes it, and '{' opens a
// complex (nested) value.  Lines starting with '#' are comments.
std::vector<Setting> from_string(const std::string& raw) {
  std::string data;
  {
    std::istringstream in(raw);
    std::string line;
    while (std::getline(in, line)) {
      const std::string t = trim(line);
      if (!t.empty() && t[0] == '#') continue;
      data += line;
      data += '\n';
    }
  }
  std::vector<Setting> out;
  size_t start = 0;
  while (start < data.size()) {
    const size_t match = data.find(':', start);
    if (match == std::string::npos) break;
    Setting s;
    s.name = data.substr(start, match - start);
    remove_chars(s.name, " {\n\t\r");
    size_t i = match + 1;
    int depth = 0;
    bool done = false;
    while (i < data.size() && !done) {
      const char c = data[i++];
      if (c == '{') {
        ++depth;
        s.complex = true;
      } else if (c == '}') {
        if (depth == 0) done = true;
        else if (--depth == 0 && s.complex) {
          // the closing brace of this value: take the separator after it
          while (i < data.size() && (data[i] == ' ' || data[i] == '\n' || data[i] == '\t')) ++i;
          if (i < data.size() && data[i] == ',') ++i;
          done = true;
        }
      } else if (c == ',' && depth == 0) {
        done = true;
      }
    }
    s.value = data.substr(match + 1, i - match - 1);
    out.push_back(s);
    start = i;
  }
  return out;
}

int parse_simulator(const std::string& text, uint32_t* policy, int32_t* dims) {
  // SimTraits defaults (simulator/simulator_traits.hpp:44-58): double, 1-D,
  // ideal gas, conservative form, Superbee, MUSCL-Hancock, FORCE
  uint32_t pol = FL_DTYPE_F64 | FL_LIMITER_SUPERBEE | FL_RECON_MUSCL | FL_FLUX_FORCE;
  int d = 1;
  bool found = false;
  for (const Setting& top : from_string(text)) {
    if (top.name != "simulator") continue;
    found = true;
    std::string inner = top.value;
    const size_t a = inner.find('{'), b = inner.rfind('}');
    if (a == std::string::npos || b == std::string::npos || b < a)
      return fl::set_error(fl::kEInval, "simulator setting must be { name : value, ... }");
    inner = inner.substr(a + 1, b - a - 1);
    for (Setting s : from_string(inner)) {
      if (s.complex)
        return fl::set_error(fl::kEInval, "simulator setting '%s' must be a plain value",
                             s.name.c_str());
      remove_chars(s.value, ",}\n");
      const std::string v = trim(s.value);
      const std::string& n = s.name;
      auto bad = [&]() {
        return fl::set_error(fl::kEInval, "unsupported %s '%s'", n.c_str(), v.c_str());
      };
      if (n == "data_type") {
        if (v == "double") pol = (pol & ~1u) | FL_DTYPE_F64;
        else if (v == "float") pol = (pol & ~1u) | FL_DTYPE_F32;
        else return bad();
      } else if (n == "dimensions") {
        if (v == "one") d = 1;
        else if (v == "two") d = 2;
        else if (v == "three") d = 3;
        else return bad();
      } else if (n == "limit_form") {
        if (v != "conservative") return bad();   // the primitive form is not built
      } else if (n == "limiter") {
        if (v == "van-leer") pol = (pol & ~(1u << 3)) | FL_LIMITER_VANLEER;
        else if (v == "superbee") pol = (pol & ~(1u << 3)) | FL_LIMITER_SUPERBEE;
        else return bad();                       // void / linear are not built
      } else if (n == "material") {
        if (v != "ideal-gas") return bad();
      } else if (n == "reconstructor") {
        if (v == "muscl-hancock") pol = (pol & ~(1u << 4)) | FL_RECON_MUSCL;
        else if (v == "none") pol = (pol & ~(1u << 4)) | FL_RECON_BASIC;
        else return bad();
      } else if (n == "flux_method") {
        uint32_t f;
        if (v == "force") f = FL_FLUX_FORCE;
        else if (v == "hllc") f = FL_FLUX_HLLC;
        else if (v == "lax-friedrichs") f = FL_FLUX_LF;
        else if (v == "richtmyer") f = FL_FLUX_RICHTMYER;
        else return bad();
        pol = (pol & ~(3u << 1)) | f;
      } else if (n == "solve_method") {
        if (v != "split") return bad();          // the reference's unsplit solver is unfinished
      } else if (n == "execution") {
        if (v != "gpu") return bad();
      } else {
        return fl::set_error(fl::kEInval, "unknown simulator setting '%s'", n.c_str());
      }
    }
  }
  if (!found) return fl::set_error(fl::kEInval, "no 'simulator : { ... }' setting");
  *policy = pol;
  *dims = d;
  return fl::kOk;
}

}  // namespace

extern "C" {

int fl_policy_from_settings(const char* text, uint32_t* policy, int32_t* dims) {
  if (text == nullptr || policy == nullptr || dims == nullptr)
    return fl::set_error(fl::kEInval, "NULL argument");
  return parse_simulator(std::string(text), policy, dims);
}

int fl_policy_from_settings_file(const char* path, uint32_t* policy, int32_t* dims) {
  if (path == nullptr || policy == nullptr || dims == nullptr)
    return fl::set_error(fl::kEInval, "NULL argument");
  std::ifstream f(path);
  if (!f) return fl::set_error(fl::kEInval, "cannot open settings file '%s'", path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_simulator(ss.str(), policy, dims);
}

}  // extern "C"
