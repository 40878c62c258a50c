// Host check of gnufft::fftcore::FastDiv (the multiply-shift division of
// the transform passes' tile, job and unit indices) against integer
// division: divisors 1..5000, powers of two and their neighbours, random
// divisors below 2^31; dividends at the edges (0, 1, d - 1, d, d + 1,
// 2^31 - 1) and random below 2^31.  Prints "failures N".
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "fftcore.cuh"

int main()
{
  using gnufft::fftcore::FastDiv;
  std::vector<uint32_t> divs;
  for (uint32_t d = 1; d <= 5000; ++d)
    divs.push_back(d);
  for (int k = 0; k < 31; ++k)
  {
    divs.push_back(1u << k);
    divs.push_back((1u << k) + 1u);
    if (k > 0)
      divs.push_back((1u << k) - 1u);
  }
  divs.push_back(0x7FFFFFFFu);
  std::mt19937 rng(12345);
  std::uniform_int_distribution<uint32_t> any(1u, 0x7FFFFFFFu);
  for (int i = 0; i < 3000; ++i)
    divs.push_back(any(rng));
  long long failures = 0, checks = 0;
  for (uint32_t d : divs)
  {
    const FastDiv f(d);
    std::vector<uint32_t> ns = {0u, 1u, d - 1u, d, d + 1u, 0x7FFFFFFFu,
                                0x7FFFFFFEu};
    for (int i = 0; i < 400; ++i)
      ns.push_back(any(rng) - 1u);
    for (uint32_t n : ns)
    {
      if (n > 0x7FFFFFFFu)
        continue;  // the contract: dividends below 2^31
      ++checks;
      if (f.div(n) != n / d)
      {
        if (failures < 10)
          std::printf("mismatch d=%u n=%u got %u want %u\n", d, n, f.div(n),
                      n / d);
        ++failures;
      }
    }
  }
  std::printf("checks %lld\nfailures %lld\n", checks, failures);
  return failures != 0;
}
