// NB resampling of a GLM null fit with the C++ standard library's own
// distributions, as the reference's GLM permutations draw it
// (include/eqtl/scan_cis.hpp:106-127): for each seed, std::mt19937(seed)
// first shuffles an index vector of n entries (std::shuffle; the result is
// not used), then draws y_i ~ Poisson(Gamma(1/phi, phi mu_i)) in sample
// order (Poisson(mu_i) when phi <= 1e-9, 0 when mu_i <= 1e-12).
// stdin: n phi, the n means, the number of seeds, the seeds.
// stdout: one line of n counts per seed. Test infrastructure only.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

int main() {
  int n = 0;
  double phi = 0;
  if (std::scanf("%d %lf", &n, &phi) != 2 || n <= 0) return 1;
  std::vector<double> mu(static_cast<size_t>(n));
  for (double& m : mu)
    if (std::scanf("%lf", &m) != 1) return 1;
  int k = 0;
  if (std::scanf("%d", &k) != 1) return 1;
  for (int s = 0; s < k; ++s) {
    unsigned long seed = 0;
    if (std::scanf("%lu", &seed) != 1) return 1;
    std::mt19937 rng(static_cast<unsigned>(seed));
    std::vector<int> idx(static_cast<size_t>(n));
    std::iota(idx.begin(), idx.end(), 0);
    std::shuffle(idx.begin(), idx.end(), rng);
    for (int i = 0; i < n; ++i) {
      const double m = mu[static_cast<size_t>(i)];
      long y = 0;
      if (m > 1e-12) {
        if (phi > 1e-9) {
          std::gamma_distribution<double> gam(1.0 / phi, phi * m);
          std::poisson_distribution<long> pois(gam(rng));
          y = pois(rng);
        } else {
          std::poisson_distribution<long> pois(m);
          y = pois(rng);
        }
      }
      std::printf(i ? " %ld" : "%ld", y);
    }
    std::printf("\n");
  }
  return 0;
}
