#include "header.hpp"
#include "lyotropic_gpu.hpp"
#include "error_msg.hpp"
#include "random.hpp"

#include <cmath>

using namespace std;
namespace opt = boost::program_options;

// from the driver (src/main.cpp of the reference, or the standalone driver)
extern unsigned nsubsteps;

LyotropicGPU::LyotropicGPU(unsigned LX_, unsigned LY_, unsigned BC_)
{
  // Grid geometry without the CPU neighbour tables: the device owns the
  // lattice, so only the sizes are recorded here.
  LX = LX_;
  LY = LY_;
  BC = BC_;
  Type = BC_ == 0 ? GridType::Periodic : GridType::Layer;
  DomainSize = LX*LY;
  TotalSize = BC_ == 0 ? DomainSize : (LX + 2)*(LY + 2);
}

LyotropicGPU::~LyotropicGPU()
{
  mass_lb_destroy(lattice);
}

void LyotropicGPU::Initialize()
{
  angle = angle_deg*M_PI/180.;
  if(nsubsteps > 1)
    throw error_msg("time stepping not implemented for this model"
                    ", please set nsubsteps=1.");
  const int prec = mass_gpu::precision_code(precision);
  if(prec < 0)
    throw error_msg("precision '", precision, "' unknown (fp32 or fp64).");

  const size_t N = DomainSize;
  ff.assign(N, mass_gpu::Node{});
  for(auto* f : {&QQxx, &QQyx, &phi, &sigmaXX, &sigmaYY, &sigmaYX, &sigmaXY,
                 &sigma_bulk, &sigma_elastic_xx, &sigma_elastic_yx,
                 &sigma_phase_field_xx, &sigma_phase_field_yx,
                 &sigma_active_xx, &sigma_active_yx})
    f->assign(N, 0.);

  mass_lb_params p{};
  p.model = DeviceModel();
  p.GammaQ = GammaQ; p.GammaP = GammaP; p.xi = xi; p.tauNem = tauNem;
  p.tauIso = tauIso; p.rho = rho; p.friction = friction; p.AA = AA; p.CC = CC;
  p.LL = LL; p.KK = KK; p.zeta = zeta; p.zetaI = zetaI; p.conc = conc;
  p.npc = npc;
  mass_lb_destroy(lattice);
  lattice = nullptr;
  const int r = mass_lb_create(&p, LX, LY, BC, prec, &lattice);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_create", r));
}

void LyotropicGPU::ConfigureAtNode(unsigned k)
{
  using mass_gpu::udiff;
  using mass_gpu::uwrap;
  double nematicOrder = 0;
  const unsigned x = GetXPosition(k);
  const unsigned y = GetYPosition(k);
  const double r2 = radius*radius;
  bool random_everywhere = false;
  double p_value = 0;
  auto sq = [](double a) { return a*a; };

  if(init_config == "circle")
  {
    if(sq(udiff(x, LX/2)) + sq(udiff(y, LY/2)) <= r2) nematicOrder = 1;
  }
  else if(init_config == "square")
  {
    if(udiff(LY/2, y) < level/2 && udiff(LX/2, x) < level/2) nematicOrder = 1;
  }
  else if(init_config == "stripe")
  {
    if(udiff(LY/2, y) < level/2) nematicOrder = 1;
  }
  else if(init_config == "half")
  {
    if(y < level) nematicOrder = 1;
  }
  else if(init_config == "boxatwall")
  {
    if(BC == 201 || BC == 501 || BC == 4)
    {
      if(x < level && udiff(LY/2, y) < level/2) nematicOrder = 1;
    }
    else if(y < level && udiff(LX/2, x) < level) nematicOrder = 1;
  }
  else if(init_config == "cuttingatwall")
  {
    if(BC == 201 || BC == 501 || BC == 4)
    {
      const unsigned up = LY/2 + int(radius*1.5), dn = LY/2 - int(radius*1.5);
      if(sq(x) + sq(uwrap(udiff(y, up), LY)) <= r2) nematicOrder = 1;
      if(sq(x) + sq(uwrap(udiff(y, dn), LY)) <= r2) nematicOrder = 1;
    }
    else if(y < level && udiff(LX/2, x) < level) nematicOrder = 1;
  }
  else if(init_config == "circleatwall")
  {
    if(BC == 201 || BC == 501)
    {
      if(sq(x) + sq(uwrap(udiff(y, LY/2), LY)) <= r2) nematicOrder = 1;
    }
    else if(sq(uwrap(udiff(x, LX/2), LX)) + sq(y) <= r2) nematicOrder = 1;
  }
  else if(init_config == "wettedwall")
  {
    if(BC == 201 || BC == 501) { if(x < level) nematicOrder = 1; }
    else if(y < level) nematicOrder = 1;
  }
  else if(init_config == "random-disk")
  {
    // S = 1 everywhere; phi a tanh disk of radius `radius` centred at
    // (LX/2, LY/2): phi = (1 - tanh((r - radius)/width))/2
    random_everywhere = true;
    const double dx = double(x) - LX/2., dy = double(y) - LY/2.;
    p_value = .5*(1. - tanh((sqrt(dx*dx + dy*dy) - radius)/width));
  }
  else if(init_config == "random-phi")
  {
    // S = 1 everywhere; phi ~ N(conc, phi_sd) i.i.d. (drawn after the angle)
    random_everywhere = true;
  }
  else
    throw error_msg("error: initial configuration '", init_config, "' unknown.");

  const double theta = angle + noise*M_PI*(random_real() - .5);
  if(random_everywhere)
  {
    QQxx[k] = cos(2*theta);
    QQyx[k] = sin(2*theta);
    phi[k] = init_config == "random-phi" ? conc + random_normal(phi_sd) : p_value;
  }
  else
  {
    QQxx[k] = nematicOrder*(cos(2*theta));
    QQyx[k] = nematicOrder*(sin(2*theta));
    phi[k] = nematicOrder*conc;
  }
  totalphi += phi[k];
  ff[k] = mass_gpu::equilibrium(0, 0, rho);
  for(double f : ff[k]) ftot += f;
  ptot += phi[k];
}

void LyotropicGPU::Configure()
{
  totalphi = ftot = ptot = 0;
  for(unsigned k = 0; k < DomainSize; ++k) ConfigureAtNode(k);
  std::vector<double> flat;
  mass_gpu::flatten(ff, flat);
  const int r = mass_lb_upload(lattice, flat.data(), QQxx.data(), QQyx.data(), phi.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_upload", r));
  steps_done = 0;
}

void LyotropicGPU::Step()
{
  // Step() must not throw (src/models.hpp:81-86): a failure is kept and
  // reported by the next RuntimeChecks().
  if(!step_error.empty()) return;
  const int r = mass_lb_step(lattice, 1);
  if(r != MASS_LB_OK) step_error = mass_gpu::abi_error("mass_lb_step", r);
  else ++steps_done;
}

void LyotropicGPU::SyncFrame()
{
  std::vector<double> flat(9*static_cast<size_t>(DomainSize));
  int r = mass_lb_download(lattice, MASS_LB_FF, flat.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_download", r));
  mass_gpu::unflatten(flat, ff);
  struct { int id; std::vector<double>* f; } fields[] = {
    {MASS_LB_QQXX, &QQxx}, {MASS_LB_QQYX, &QQyx}, {MASS_LB_PHI, &phi},
    {MASS_LB_SIGMAXX, &sigmaXX}, {MASS_LB_SIGMAXY, &sigmaXY},
    {MASS_LB_SIGMAYX, &sigmaYX}, {MASS_LB_SIGMAYY, &sigmaYY},
    {MASS_LB_SIGMA_BULK, &sigma_bulk}, {MASS_LB_SIGMA_ELASTIC_XX, &sigma_elastic_xx},
    {MASS_LB_SIGMA_ELASTIC_YX, &sigma_elastic_yx},
    {MASS_LB_SIGMA_PHASE_FIELD_XX, &sigma_phase_field_xx},
    {MASS_LB_SIGMA_PHASE_FIELD_YX, &sigma_phase_field_yx},
    {MASS_LB_SIGMA_ACTIVE_XX, &sigma_active_xx},
    {MASS_LB_SIGMA_ACTIVE_YX, &sigma_active_yx}};
  for(auto& f : fields)
  {
    // before the first step the stresses are still the zeros the reference
    // holds at that point
    if(f.id >= MASS_LB_N && steps_done == 0) continue;
    r = mass_lb_download(lattice, f.id, f.f->data());
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_download", r));
  }
}

void LyotropicGPU::RuntimeChecks()
{
  if(!step_error.empty()) throw error_msg(step_error);
  double fcheck = 0, pcheck = 0;
  int bad = 0;
  const int r = mass_lb_checks(lattice, &fcheck, &pcheck, &bad);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_checks", r));
  cout << "fcheck: " << fcheck << "/" << ftot << '\n';
  if(bad) throw error_msg("nan found in the lattice state.");
  if(abs(ftot - fcheck) > 1)
    throw error_msg("f is not conserved (", ftot, "/", fcheck, ")");
  cout << "pcheck: " << pcheck << "/" << ptot << '\n';
}

option_list LyotropicGPU::GetOptions()
{
  opt::options_description model_options("Model options");
  model_options.add_options()
    ("GammaQ", opt::value<double>(&GammaQ), "Q-tensor mobility")
    ("GammaP", opt::value<double>(&GammaP), "binary mobility")
    ("xi", opt::value<double>(&xi), "tumbling/aligning parameter")
    ("tauNem", opt::value<double>(&tauNem), "nematic viscosity")
    ("tauIso", opt::value<double>(&tauIso), "isotropic viscosity")
    ("rho", opt::value<double>(&rho), "fluid density")
    ("friction", opt::value<double>(&friction), "friction from confinement")
    ("AA", opt::value<double>(&AA), "binary fluid bulk constant")
    ("CC", opt::value<double>(&CC), "coupling constant")
    ("LL", opt::value<double>(&LL), "elastic constant")
    ("KK", opt::value<double>(&KK), "binary gradient constant")
    ("zeta", opt::value<double>(&zeta), "activity parameter")
    ("zetaI", opt::value<double>(&zetaI), "activity isotropic parameter")
    ("npc", opt::value<unsigned>(&npc),
     "number of correction steps for the predictor-corrector method");

  opt::options_description config_options("Initial configuration options");
  config_options.add_options()
    ("config", opt::value<string>(&init_config), "initial configuration")
    ("level", opt::value<double>(&level), "starting thickness of the nematic region")
    ("conc", opt::value<double>(&conc), "starting phi concentration of nematic region")
    ("radius", opt::value<double>(&radius), "radius of the initial circle")
    ("angle", opt::value<double>(&angle_deg), "initial angle to x direction (in degrees)")
    ("noise", opt::value<double>(&noise), "size of initial variations")
    ("width", opt::value<double>(&width),
     "interface width of the tanh disk (config=random-disk)")
    ("phi_sd", opt::value<double>(&phi_sd),
     "standard deviation of phi around conc (config=random-phi)");

  opt::options_description gpu_options("GPU options");
  gpu_options.add_options()
    ("precision", opt::value<string>(&precision),
     "fp32 (fused sm_100a kernel) or fp64 (bit-exact with the CPU model)");

  return { model_options, config_options, gpu_options };
}
