// LyotropicGPU: the MASS lyotropic model (reference src/models/lyotropic.hpp)
// with its time step on a B200 through include/mass_lb.h.
//
// Drop-in contract kept from the reference model:
//  * constructed by declare_model's factory as (LX, LY, BC);
//  * the same runcard options (GetOptions, src/models/lyotropic.cpp:551-602)
//    plus new ones: "precision" (fp32 | fp64), "width" (tanh interface
//    width of the "random-disk" configuration) and "phi_sd";
//  * the same Initialize / Configure / Step / RuntimeChecks life cycle and
//    error messages;
//  * serialize_params / serialize_frame with the reference's member names in
//    the reference's order (src/models/lyotropic.hpp:94-138), so
//    parameters.json and frame<t>.json have the same schema.
// The device holds the state; the host copies below are refreshed when a
// frame is serialized.
#ifndef MODELS_LYOTROPIC_GPU_HPP_
#define MODELS_LYOTROPIC_GPU_HPP_

#include "models.hpp"
#include "gpu_common.hpp"

class LyotropicGPU : public Model
{
protected:
  /** runcard parameters (reference names) */
  double GammaP = 0, GammaQ = 0, xi = 0, tauNem = 0, tauIso = 0, friction = 0;
  double LL = 0, KK = 0, AA = 0, CC = 0, zeta = 0, zetaI = 0;
  double rho = 40.;
  unsigned npc = 1;
  std::string init_config;
  double level = 0, conc = 0, angle_deg = 0, angle = 0, noise = 0, radius = 0;
  /** options of this model: device precision, tanh width, phi noise */
  std::string precision = "fp32";
  double width = 2., phi_sd = 0.;
  /** totals for the runtime checks (src/models/lyotropic.hpp:31-44) */
  double totalphi = 0., ftot = 0, ptot = 0;

  mass_lb_handle* lattice = nullptr;
  std::string step_error;      // first failure of Step(), reported by RuntimeChecks
  unsigned long long steps_done = 0;

  /** Refresh the host frame fields from the device. */
  void SyncFrame();
  /** mass_lb_model of the device lattice this class creates */
  virtual int DeviceModel() const { return MASS_LB_LYOTROPIC; }

public:
  LyotropicGPU(unsigned LX, unsigned LY, unsigned BC);
  virtual ~LyotropicGPU();

  /** frame fields (host copies) */
  std::vector<mass_gpu::Node> ff;
  std::vector<double> QQxx, QQyx, phi;
  std::vector<double> sigmaXX, sigmaYY, sigmaYX, sigmaXY;
  std::vector<double> sigma_bulk, sigma_elastic_xx, sigma_elastic_yx,
    sigma_phase_field_xx, sigma_phase_field_yx, sigma_active_xx, sigma_active_yx;

  /** the reference's per-site initial state (src/models/lyotropic.cpp:69-160)
   * extended with "random-disk" and "random-phi" */
  virtual void ConfigureAtNode(unsigned);

  virtual void Initialize();
  virtual void Configure();
  virtual void Step();
  virtual void RuntimeChecks();
  virtual option_list GetOptions();

  /** handle of the device lattice (for tools built on this model) */
  mass_lb_handle* device_lattice() { return lattice; }

  template<class Archive>
  void serialize_params(Archive& ar)
  {
    ar & auto_name(level)
       & auto_name(conc)
       & auto_name(angle)
       & auto_name(noise)
       & auto_name(totalphi)
       & auto_name(rho)
       & auto_name(GammaP)
       & auto_name(GammaQ)
       & auto_name(xi)
       & auto_name(zeta)
       & auto_name(zetaI)
       & auto_name(tauNem)
       & auto_name(tauIso)
       & auto_name(friction)
       & auto_name(LL)
       & auto_name(KK)
       & auto_name(init_config)
       & auto_name(AA)
       & auto_name(CC);
  }

  template<class Archive>
  void serialize_frame(Archive& ar)
  {
    SyncFrame();
    ar & auto_name(ff)
       & auto_name(QQxx)
       & auto_name(QQyx)
       & auto_name(phi)
       & auto_name(sigmaXX)
       & auto_name(sigmaXY)
       & auto_name(sigmaYX)
       & auto_name(sigmaYY)
       & auto_name(sigma_bulk)
       & auto_name(sigma_elastic_xx)
       & auto_name(sigma_elastic_yx)
       & auto_name(sigma_phase_field_xx)
       & auto_name(sigma_phase_field_yx)
       & auto_name(sigma_active_xx)
       & auto_name(sigma_active_yx);
  }
};

#endif
