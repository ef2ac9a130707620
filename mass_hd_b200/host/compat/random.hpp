// Global pseudo-random stream of the MASS models: std::mt19937 with
// uniform_real_distribution / normal_distribution, reseeded by set_seed
// (reference: src/random.cpp:12-45). Using the same standard-library
// engines gives the same draws as the reference for the same seed.
#ifndef MASS_GPU_COMPAT_RANDOM_HPP_
#define MASS_GPU_COMPAT_RANDOM_HPP_

double random_real(double min = 0., double max = 1.);
double random_normal(double sigma = 1.);
unsigned randu();
void set_seed(unsigned);

#endif
