// Device-side division / death masks (masks.cu).
#pragma once

#include <cuda_runtime.h>

namespace mlb {

// phi of a lattice as the step kernels hold it: plane with ghost ring g and
// row stride EY (FP64 / FP32 unfused), or g = 0, EY = LY (FP32 fused)
template<typename T>
struct MaskView
{
  const T* phi;
  int LX, LY, g, EY;
};

struct MaskScratch
{
  int* block_cnt = nullptr;        // candidates per block of 1024 sites
  long long* block_off = nullptr;  // exclusive offsets
  long long* total = nullptr;      // number of candidates
  unsigned char* center = nullptr; // LX*LY, site order
  unsigned char* mask[2] = {nullptr, nullptr};   // division, death (LX*LY)
  double* draws = nullptr;         // the caller's uniforms
  long long draws_cap = 0;
};

// Uniforms supplied ahead by the caller, consumed on the device: a ring of
// `cap` doubles, `head` (device) = draws taken so far, `supplied` = draws
// written so far (host-side count, passed to the kernels by value).
struct MaskQueue
{
  double* buf = nullptr;
  long long cap = 0;
  long long* head = nullptr;
  long long supplied = 0;
};

// One queued draw: which masks, their coefficients and the source plane.
template<typename T>
struct QueuedDraw
{
  int kinds;             // bit 0 division, bit 1 death
  double coef[2];        // division, death
  double radius[2];
  double phi_critical;
  double alpha, beta;
  T* src;                // the step kernels' source plane (ghost ring g, row stride EY)
  int g, EY;
  int* err;
  long long* snap;       // after the draw: [0] queue head, [1] error flag
};

int mask_blocks(long long nsites);

template<typename T>
cudaError_t mask_count(const MaskView<T>& v, const MaskScratch& s, cudaStream_t st);
template<typename T>
cudaError_t mask_draw(const MaskView<T>& v, const MaskScratch& s, int kind, long long ndraws,
                      double coef, double phi_critical, double radius, cudaStream_t st);
// A whole queued draw in one cooperative launch: count, offsets, centres of
// both kinds, circles, source plane and head advance, with grid barriers
// between the phases.
template<typename T>
cudaError_t mask_draw_queued_fused(const MaskView<T>& v, const MaskScratch& s, const MaskQueue& q,
                                   const QueuedDraw<T>& w, cudaStream_t st);
template<typename T>
cudaError_t mask_rate(int LX, int LY, int g, int EY, const MaskScratch& s, double alpha,
                      double beta, T* src, cudaStream_t st);

} // namespace mlb
