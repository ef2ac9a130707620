// NematicGPU: the MASS nematic model (reference src/models/nematic.hpp) with
// its time step on a B200 through include/mass_lb.h. Same runcard options
// (src/models/nematic.cpp:409-445) plus "precision"; same serialized
// parameters and frame fields (src/models/nematic.hpp:84-108). Thermal
// fluctuations (Q_kBT, u_kBT != 0) are rejected by Initialize().
#ifndef MODELS_NEMATIC_GPU_HPP_
#define MODELS_NEMATIC_GPU_HPP_

#include "models.hpp"
#include "gpu_common.hpp"

class NematicGPU : public Model
{
protected:
  double angle_deg = 0, angle = 0, noise = 0;
  double rho = 40.;
  double Gamma = 0, xi = 0, tau = 0, friction = 0, LL = 0, CC = 0, zeta = 0;
  double Q_kBT = 0, u_kBT = 0;
  unsigned npc = 1;
  std::string precision = "fp32";
  double ftot = 0;

  mass_lb_handle* lattice = nullptr;
  std::string step_error;

  void SyncFrame();

public:
  NematicGPU(unsigned LX, unsigned LY, unsigned BC);
  virtual ~NematicGPU();

  std::vector<mass_gpu::Node> ff;
  std::vector<double> QQxx, QQyx;

  virtual void ConfigureAtNode(unsigned);
  virtual void Initialize();
  virtual void Configure();
  virtual void Step();
  virtual void RuntimeChecks();
  virtual option_list GetOptions();

  mass_lb_handle* device_lattice() { return lattice; }

  template<class Archive>
  void serialize_params(Archive& ar)
  {
    ar & auto_name(angle)
       & auto_name(noise)
       & auto_name(rho)
       & auto_name(Gamma)
       & auto_name(xi)
       & auto_name(zeta)
       & auto_name(tau)
       & auto_name(friction)
       & auto_name(LL)
       & auto_name(CC);
  }

  template<class Archive>
  void serialize_frame(Archive& ar)
  {
    SyncFrame();
    ar & auto_name(ff)
       & auto_name(QQxx)
       & auto_name(QQyx);
  }
};

#endif
