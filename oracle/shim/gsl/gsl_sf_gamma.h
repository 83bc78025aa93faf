// Test infrastructure only: the one GSL special function src/stats_extra.cpp
// calls (GSL is not installed in this image). ln B(a,b) from std::lgamma.
#pragma once
#include <cmath>

inline double gsl_sf_lnbeta(double a, double b) {
  return std::lgamma(a) + std::lgamma(b) - std::lgamma(a + b);
}
