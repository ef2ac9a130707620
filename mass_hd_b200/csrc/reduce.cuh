// Conservation sums for Model::RuntimeChecks (src/models/lyotropic.cpp:527-549).
#pragma once

#include "lb_common.cuh"

namespace mlb {

// Where the populations and phi of one lattice live on the device.
template<typename T>
struct SumView
{
  const T* ff;          // 9 planes, plane v at ff + v*plane
  const T* Qxx;
  const T* Qyx;
  const T* phi;         // may be null (nematic)
  long long plane;      // plane stride (elements)
  int LX, LY, g, EY;    // domain and extended-row geometry
  double rest;          // value added per site to the population sum
                        // (rho for deviation storage, else 0)
};

// Number of partial-sum slots launch_sums needs in `scratch` (doubles).
int sums_scratch_doubles();

// Kahan-Babuska sums of all populations and of phi over the domain, plus a
// non-finite flag over ff, Q and phi. Results (fsum, phisum, flag as double)
// land in out[0..2] (device memory). `scratch` holds sums_scratch_doubles()
// doubles of device memory, overwritten.
cudaError_t launch_sums_f64(const SumView<double>& v, double* scratch,
                            double* out, cudaStream_t st);
cudaError_t launch_sums_f32(const SumView<float>& v, double* scratch,
                            double* out, cudaStream_t st);

} // namespace mlb
