// FP64 host DFT used at context set-up to turn frequency responses into
// time-domain kernels (recursive mixed-radix decimation in time; sizes with
// prime factors 2, 3, 5, 7, other primes fall back to direct sums).
#pragma once
#include <complex>
#include <vector>

namespace cuvhs {

using cd = std::complex<double>;

// Unnormalised DFT of length n = x.size(); sign -1 forward, +1 inverse.
std::vector<cd> host_dft(const std::vector<cd>& x, int sign);

}  // namespace cuvhs
