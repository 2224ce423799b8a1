// wih_analytic_integral_audit: drop-in for the reference's audit reader
// (benchmarks/submission_study/analytic_integral_audit.cpp), which the
// quadrature check benchmarks/matched_accuracy/check_integral.py drives:
// reads "d r R A" records from stdin until the input ends and prints, one
// per line at 17 significant digits, the exact ball integral of the bump
// A (1 - |x-c|^2/R^2)_+^2 centred at distance d from a ball of radius r
// (the EXACT source's closed form), evaluated on the GPU
// (twos_ball_green_integral).  Errors print to stderr and return 1.
#include <iomanip>
#include <iostream>
#include <vector>

#include "twos.h"

int main() {
  std::vector<double> cases;
  double d, r, R, A;
  while (std::cin >> d >> r >> R >> A) {
    cases.push_back(d);
    cases.push_back(r);
    cases.push_back(R);
    cases.push_back(A);
  }
  const uint32_t n = static_cast<uint32_t>(cases.size() / 4);
  std::vector<double> out(n);
  if (twos_ball_green_integral(cases.data(), n, out.data(), 0) != TWOS_OK) {
    std::cerr << twos_last_error() << '\n';
    return 1;
  }
  std::cout << std::setprecision(17);
  for (double v : out) std::cout << v << '\n';
  return 0;
}
