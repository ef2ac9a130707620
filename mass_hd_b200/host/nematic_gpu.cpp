#include "header.hpp"
#include "nematic_gpu.hpp"
#include "error_msg.hpp"
#include "random.hpp"

#include <cmath>

using namespace std;
namespace opt = boost::program_options;

extern unsigned nsubsteps;

NematicGPU::NematicGPU(unsigned LX_, unsigned LY_, unsigned BC_)
{
  LX = LX_;
  LY = LY_;
  BC = BC_;
  Type = BC_ == 0 ? GridType::Periodic : GridType::Layer;
  DomainSize = LX*LY;
  TotalSize = BC_ == 0 ? DomainSize : (LX + 2)*(LY + 2);
}

NematicGPU::~NematicGPU()
{
  mass_lb_destroy(lattice);
}

void NematicGPU::Initialize()
{
  angle = angle_deg*M_PI/180.;
  if(nsubsteps > 1)
    throw error_msg("time stepping not implemented for this model"
                    ", please set nsubsteps=1.");
  if(Q_kBT != 0 || u_kBT != 0)
    throw error_msg("thermal fluctuations (Q_kBT, u_kBT) are not available in "
                    "the GPU nematic model; set both to 0.");
  const int prec = mass_gpu::precision_code(precision);
  if(prec < 0)
    throw error_msg("precision '", precision, "' unknown (fp32 or fp64).");

  ff.assign(DomainSize, mass_gpu::Node{});
  QQxx.assign(DomainSize, 0.);
  QQyx.assign(DomainSize, 0.);

  mass_lb_params p{};
  p.model = MASS_LB_NEMATIC;
  p.GammaQ = Gamma; p.xi = xi; p.tauNem = tau; p.tauIso = tau; p.rho = rho;
  p.friction = friction; p.CC = CC; p.LL = LL; p.zeta = zeta; p.npc = npc;
  mass_lb_destroy(lattice);
  lattice = nullptr;
  const int r = mass_lb_create(&p, LX, LY, BC, prec, &lattice);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_create", r));
}

void NematicGPU::ConfigureAtNode(unsigned k)
{
  // src/models/nematic.cpp:55-68
  const double theta = angle + noise*M_PI*(random_real() - .5);
  QQxx[k] = cos(2*theta);
  QQyx[k] = sin(2*theta);
  ff[k] = mass_gpu::equilibrium(0, 0, rho);
  for(double f : ff[k]) ftot += f;
}

void NematicGPU::Configure()
{
  ftot = 0;
  for(unsigned k = 0; k < DomainSize; ++k) ConfigureAtNode(k);
  std::vector<double> flat;
  mass_gpu::flatten(ff, flat);
  const int r = mass_lb_upload(lattice, flat.data(), QQxx.data(), QQyx.data(), nullptr);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_upload", r));
}

void NematicGPU::Step()
{
  if(!step_error.empty()) return;
  const int r = mass_lb_step(lattice, 1);
  if(r != MASS_LB_OK) step_error = mass_gpu::abi_error("mass_lb_step", r);
}

void NematicGPU::SyncFrame()
{
  std::vector<double> flat(9*static_cast<size_t>(DomainSize));
  int r = mass_lb_download(lattice, MASS_LB_FF, flat.data());
  if(r == MASS_LB_OK) r = mass_lb_download(lattice, MASS_LB_QQXX, QQxx.data());
  if(r == MASS_LB_OK) r = mass_lb_download(lattice, MASS_LB_QQYX, QQyx.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_download", r));
  mass_gpu::unflatten(flat, ff);
}

void NematicGPU::RuntimeChecks()
{
  // src/models/nematic.cpp:397-407
  if(!step_error.empty()) throw error_msg(step_error);
  double fcheck = 0;
  int bad = 0;
  const int r = mass_lb_checks(lattice, &fcheck, nullptr, &bad);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_checks", r));
  if(bad) throw error_msg("nan found in the lattice state.");
  if(abs(ftot - fcheck) > 1)
    throw error_msg("f is not conserved (", ftot, "/", fcheck, ")");
}

option_list NematicGPU::GetOptions()
{
  opt::options_description model_options("Model options");
  model_options.add_options()
    ("Gamma", opt::value<double>(&Gamma), "Mobility")
    ("xi", opt::value<double>(&xi), "tumbling/aligning parameter")
    ("tau", opt::value<double>(&tau), "viscosity")
    ("rho", opt::value<double>(&rho), "fluid density")
    ("Q_kBT", opt::value<double>(&Q_kBT), "hydrodynamic fluctations strength")
    ("u_kBT", opt::value<double>(&u_kBT), "nematic fluctuations strength")
    ("friction", opt::value<double>(&friction), "friction")
    ("CC", opt::value<double>(&CC), "coupling constant")
    ("LL", opt::value<double>(&LL), "elastic constant")
    ("zeta", opt::value<double>(&zeta), "activity parameter")
    ("npc", opt::value<unsigned>(&npc),
     "number of correction steps for the predictor-corrector method");

  opt::options_description config_options("Initial configuration options");
  config_options.add_options()
    ("angle", opt::value<double>(&angle_deg), "initial angle to x direction (in degrees)")
    ("noise", opt::value<double>(&noise), "size of initial variations");

  opt::options_description gpu_options("GPU options");
  gpu_options.add_options()
    ("precision", opt::value<string>(&precision),
     "fp32 (fused sm_100a kernel) or fp64 (bit-exact with the CPU model)");

  return { model_options, config_options, gpu_options };
}
