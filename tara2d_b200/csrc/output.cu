// List-directed REAL(8) formatting (see output.h) and its C entry point.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "output.h"
#include "plan.h"

namespace tara {

namespace {

// one G25.17 field (Fortran G editing with an E3 exponent field)
void g_field(double x, char* field /* >= 26 bytes */) {
  char body[48];
  if (x == 0.0) {
    std::snprintf(body, sizeof body, "%s0.0000000000000000     ", std::signbit(x) ? "-" : "");
  } else {
    char m[48];
    std::snprintf(m, sizeof m, "%.16e", x);  // [-]d.dddddddddddddddde[+-]XX
    const char* e = std::strchr(m, 'e');
    const int E = std::atoi(e + 1);
    if (E >= -1 && E <= 16) {
      // F editing always writes the decimal point
      if (E == 16) std::snprintf(body, sizeof body, "%.0f.     ", x);
      else std::snprintf(body, sizeof body, "%.*f     ", 16 - E, x);
    } else {
      const int mlen = (int)(e - m);
      const int ae = std::abs(E);
      if (ae <= 999 && ae > 99)
        std::snprintf(body, sizeof body, "%.*s%c%03d", mlen, m, E < 0 ? '-' : '+', ae);
      else
        std::snprintf(body, sizeof body, "%.*sE%c%03d", mlen, m, E < 0 ? '-' : '+', ae);
    }
  }
  std::snprintf(field, 26, "%25s", body);
}

}  // namespace

void list_directed_append(std::string& out, const double* v, int n) {
  char f[32];
  for (int k = 0; k < n; k++) {
    g_field(v[k], f);
    out += ' ';
    out += f;
  }
}

}  // namespace tara

extern "C" int tara_format_list_directed(const double* v, int n, char* out, int cap) {
  if (!v || !out || n < 0 || cap < 1) return TARA_EINVAL;
  std::string s;
  tara::list_directed_append(s, v, n);
  if ((int)s.size() + 1 > cap) {
    tara::set_error("output buffer too small");
    return TARA_EINVAL;
  }
  std::memcpy(out, s.c_str(), s.size() + 1);
  return (int)s.size();
}
