// Global pseudo-random stream of the MASS models: the std::mt19937 sequence
// with uniform_real_distribution / normal_distribution, reseeded by
// set_seed (reference: src/random.cpp:12-45), so the draws are the
// reference's for the same seed. random_reals is this build's bulk form of
// n random_real() calls (the same values); the reference has no
// counterpart.
#ifndef MASS_GPU_COMPAT_RANDOM_HPP_
#define MASS_GPU_COMPAT_RANDOM_HPP_

#include <cstddef>

double random_real(double min = 0., double max = 1.);
void random_reals(double* out, std::size_t n);
double random_normal(double sigma = 1.);
unsigned randu();
void set_seed(unsigned);

#endif
