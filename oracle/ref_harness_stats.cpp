// Reference harness, partition-size report.  TEST INFRASTRUCTURE (oracle/_ref).
// Compiles calVarStdev (experiment.cpp:18-37) from the reference with a
// logger that keeps the text it is given.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>  // brings in the stream initialisation the report needs
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "ref_harness.h"

using namespace std;

namespace {
struct Logger {
  string text;
  void log(const string &s, int = 0, bool = false) { text += s + "\n"; }
};
}  // namespace

static Logger g_logger;
static Logger *logger = &g_logger;

#include "ref_stats.inc"  // generated from the reference by extract_ref.py

extern "C" int ref_cal_var_stdev(const uint64_t *sizes, int n, char *buf, int cap) {
  vector<size_t> v(sizes, sizes + n);
  g_logger.text.clear();
  calVarStdev(v);
  const string &t = g_logger.text;
  int m = (int)min<size_t>(t.size(), cap > 0 ? (size_t)cap - 1 : 0);
  if (cap > 0) {
    memcpy(buf, t.data(), m);
    buf[m] = 0;
  }
  return (int)t.size();
}
