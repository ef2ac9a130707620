// Flow and defect statistics on the device (stats.cu).
#pragma once

#include "lb_common.cuh"

namespace mlb {

constexpr int STATS_BLOCKS = 592;

template<typename T>
struct StatView
{
  const T* ff;          // 9 planes
  long long plane;
  const T* Qxx;
  const T* Qyx;
  const T* phi;         // null: no interface statistics
  int LX, LY, g, EY;    // domain and extended-row geometry
  double rest;          // added to the population sum per site (rho for deviations)
};

struct StatScratch
{
  double* U;            // 2*LX*LY: ux, uy
  double* D;            // 2*LX*LY: director nx, ny
  double* partial;      // 8*STATS_BLOCKS
  double* out;          // 5: sum u^2, sum w^2, sum w^2 (phi > .5), area, perimeter
  int* count;           // charged sites found
  int* list;            // capacity entries: k (charge > 0) or -k-1 (charge < 0)
  int capacity;
};

cudaError_t launch_stats_f64(const StatView<double>& v, const StatScratch& s, double threshold,
                             cudaStream_t st);
cudaError_t launch_stats_f32(const StatView<float>& v, const StatScratch& s, double threshold,
                             cudaStream_t st);

} // namespace mlb
