// GoOrGrowGPU: the MASS go-or-grow model (reference src/models/go-or-grow.hpp)
// with its time step on a B200 through include/mass_lb.h and
// include/mass_lb_ext.h.
//
// Same options, members and serialization order as the reference model. The
// configuration follows GoOrGrow::Configure (src/models/go-or-grow.cpp:34-40):
// the lyotropic initial state (host), the dry free-energy relaxation (device,
// mass_lb_relax_free_energy), the rest-state populations (host, uploaded),
// and the phenotype (host: the same random_normal() draws, smoothing and
// normalisation as the reference, then m = phi*chi clamped to [0, phi]).
// The division/death masks and the conserve_phi switch come from
// LyotropicWithDivisionGPU; the device turns the mask rate into the
// go-or-grow growth chi*phi*rate.
#ifndef MODELS_GO_OR_GROW_GPU_HPP_
#define MODELS_GO_OR_GROW_GPU_HPP_

#include "lyotropic_with_division_gpu.hpp"

class GoOrGrowGPU : public LyotropicWithDivisionGPU
{
protected:
  /** runcard parameters (reference names and initialisers) */
  double B = 0.;
  double Snem = 1.;
  double Dchi = 0.;
  double Achi = 0., Ochi = 0., phiswitch = 0.;
  int growTogether = 0;
  double chi0 = 0., chi_noise = 0., chi_length = 0.;
  std::string chi_config = "noise";
  unsigned relax_steps = 0;
  double relax_dt = 1.;
  int relax_phi = 0, relax_Q = 0;

  virtual int DeviceModel() const { return MASS_LB_GO_OR_GROW; }

  /** src/models/go-or-grow.cpp:42-119, on the device */
  void RelaxFreeEnergy();
  /** src/models/go-or-grow.cpp:121-141 */
  void ResetHydrodynamics();
  /** src/models/go-or-grow.cpp:143-206 */
  void ConfigurePhenotype();
  /** Refresh the host copies of m and chi from the device. */
  void SyncPhenotype();
  /** Five-point laplacian of a host field at domain site k with the
   * ghost values the reference's boundary conditions give it. */
  double HostLaplacian(const std::vector<double>& a, unsigned k) const;

public:
  GoOrGrowGPU(unsigned LX, unsigned LY, unsigned BC);

  std::vector<double> m, chi;

  virtual void Initialize();
  virtual void Configure();
  virtual option_list GetOptions();

  template<class Archive>
  void serialize_params(Archive& ar)
  {
    LyotropicWithDivisionGPU::serialize_params(ar);
    ar & auto_name(B)
       & auto_name(Snem)
       & auto_name(Dchi)
       & auto_name(Achi)
       & auto_name(Ochi)
       & auto_name(phiswitch)
       & auto_name(growTogether)
       & auto_name(chi0)
       & auto_name(chi_noise)
       & auto_name(chi_length)
       & auto_name(chi_config)
       & auto_name(relax_steps)
       & auto_name(relax_dt)
       & auto_name(relax_phi)
       & auto_name(relax_Q);
  }

  template<class Archive>
  void serialize_frame(Archive& ar)
  {
    LyotropicWithDivisionGPU::serialize_frame(ar);
    SyncPhenotype();
    ar & auto_name(m);
    ar & auto_name(chi);
  }
};

#endif
