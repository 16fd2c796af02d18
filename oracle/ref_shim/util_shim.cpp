// The handful of util.h functions (declared in the reference's util.h) that the
// reference's hot-path sources call, implemented here so those sources link without
// boost.  Used only to build the reference as a test oracle.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>

#include "util.h"

int roundUpToPowerOfTwo(int n) {
  int r = 1;
  while (r < n) r *= 2;
  return r;
}
bool isPowerOfTwo(int n) { return n == roundUpToPowerOfTwo(n); }
string pluralize(int n, const string& noun) {
  return std::to_string(n) + " " + noun + ((n == 1 || n == -1) ? "" : "s");
}
void assertFloatEq(float a, float b, const string& tag) {
  float ia = a, ib = b;
  while (a > 100) { a /= 2.0; b /= 2.0; }
  if (std::fabs(a - b) > 0.001) {
    std::cerr << tag << ": " << ia << " != " << ib << std::endl;
    std::exit(2);
  }
}
void assertFloatEq(float a, float b) { assertFloatEq(a, b, ""); }
void logErrorTimestamp() { std::cerr << "[reference oracle] "; }
void fatal(const string& message) { throw std::runtime_error(message); }
void fatal(const string& m1, const string& m2) { throw std::runtime_error(m1 + ": " + m2); }
