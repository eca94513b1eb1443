// common.cpp — shared host helpers of the CLI (reference: routines/common.cpp:4-34).
#include <algorithm>

#include "routines.h"

void flushL2() { LT_CHECK(lt_flush_l2(nullptr)); }

double envDouble(const char* name, double def) {
  const char* v = getenv(name);
  return (v != nullptr && *v != '\0') ? atof(v) : def;
}

long envLong(const char* name, long def) {
  const char* v = getenv(name);
  return (v != nullptr && *v != '\0') ? atol(v) : def;
}

double median(std::vector<double> v) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  size_t n = v.size();
  return (n % 2) ? v[n / 2] : 0.5 * (v[n / 2 - 1] + v[n / 2]);
}
