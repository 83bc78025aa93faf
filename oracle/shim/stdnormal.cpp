// Prints `count` draws of std::normal_distribution<double>(0, 1) from one
// std::mt19937(seed), one per line (%.17g): the standard library's own
// sequence, which the reference program draws its PEER starting values from
// (src/fission.cpp:226-236). Test infrastructure only: the oracle reads it to
// start its PEER restatement where the reference starts.
#include <cstdio>
#include <cstdlib>
#include <random>

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: stdnormal SEED COUNT\n");
    return 1;
  }
  std::mt19937 rng(static_cast<unsigned>(std::strtoul(argv[1], nullptr, 10)));
  std::normal_distribution<double> nd;
  const long count = std::strtol(argv[2], nullptr, 10);
  for (long i = 0; i < count; ++i) std::printf("%.17g\n", nd(rng));
  return 0;
}
