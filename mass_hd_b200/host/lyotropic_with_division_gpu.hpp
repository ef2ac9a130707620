// LyotropicWithDivisionGPU: the MASS lyotropic model with cell division and
// death (reference src/models/lyotropic-with-division.hpp) with its time step
// on a B200 through include/mass_lb.h and include/mass_lb_ext.h.
//
// Same options, members and serialization order as the reference model.
// The division and death masks follow the reference's SetMasks(): one
// random_real() per site with phi >= .5 in site order from the reference's
// generator. The host queues the generator's values on the device ahead of
// need (mass_lb_mask_supply), and the device counts the candidates, takes
// their draws, picks the centres, draws the circles and sets the source
// rate alpha*division_mask - beta*death_mask (mass_lb_draw_masks_queued). When division
// and death are off the device applies the conserve_phi correction
// (mass_lb_set_phi_conservation).
#ifndef MODELS_LYOTROPIC_WITH_DIVISION_GPU_HPP_
#define MODELS_LYOTROPIC_WITH_DIVISION_GPU_HPP_

#include "lyotropic_gpu.hpp"

class LyotropicWithDivisionGPU : public LyotropicGPU
{
protected:
  /** strengths, rates, life-times and radii (reference names) */
  double alpha = 0, beta = 0;
  double division_rate = 0, division_time = 0, division_radius = 0;
  double death_rate = 0, death_time = 0, death_radius = 0;
  double phi_critical = 1;
  unsigned division_count = 0, death_count = 0;
  bool conserve_phi = false;
  /** random_real() values handed to the device's draw queue so far. Values
   * are drawn ahead of need, in stream order, into the library's pinned
   * staging buffer; only the masks consume the generator after
   * Configure(), so every value keeps its place in the reference's stream. */
  long long supplied = 0;

  /** Redraw the masks that are due (src/models/lyotropic-with-division.cpp:35-106). */
  void SetMasks();
  /** Refresh the host copies of the masks from the device. */
  void SyncMasks();

public:
  LyotropicWithDivisionGPU(unsigned LX, unsigned LY, unsigned BC);

  std::vector<bool> division_mask, death_mask;

  virtual void Initialize();
  virtual void Configure();
  virtual void Step();
  virtual void RuntimeChecks();
  virtual option_list GetOptions();

  template<class Archive>
  void serialize_params(Archive& ar)
  {
    LyotropicGPU::serialize_params(ar);
    ar & auto_name(alpha)
       & auto_name(beta)
       & auto_name(division_rate)
       & auto_name(division_time)
       & auto_name(division_radius)
       & auto_name(death_rate)
       & auto_name(death_time)
       & auto_name(death_radius)
       & auto_name(phi_critical);
  }

  template<class Archive>
  void serialize_frame(Archive& ar)
  {
    LyotropicGPU::serialize_frame(ar);
    SyncMasks();
    ar & auto_name(division_mask)
       & auto_name(death_mask);
  }
};

#endif
