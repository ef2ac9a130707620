#include "header.hpp"
#include "go_or_grow_gpu.hpp"
#include "error_msg.hpp"
#include "random.hpp"
#include "mass_lb_ext.h"

#include <cmath>

using namespace std;
namespace opt = boost::program_options;

GoOrGrowGPU::GoOrGrowGPU(unsigned LX_, unsigned LY_, unsigned BC_)
  : LyotropicWithDivisionGPU(LX_, LY_, BC_)
{}

void GoOrGrowGPU::Initialize()
{
  LyotropicWithDivisionGPU::Initialize();

  // the reference's checks and messages (src/models/go-or-grow.cpp:17-32)
  if(chi_noise < 0)
    throw error_msg("chi-noise must be non-negative.");
  if(chi_length < 0)
    throw error_msg("chi-length must be non-negative.");
  if(relax_dt < 0)
    throw error_msg("relax-dt must be non-negative.");

  m.assign(DomainSize, 0.);
  chi.assign(DomainSize, 0.);

  mass_lb_go_or_grow_params p{};
  p.B = B; p.Snem = Snem; p.Dchi = Dchi; p.Achi = Achi; p.Ochi = Ochi;
  p.phiswitch = phiswitch; p.phi_critical = phi_critical; p.growTogether = growTogether;
  const int r = mass_lb_set_go_or_grow_params(lattice, &p);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_set_go_or_grow_params", r));
}

void GoOrGrowGPU::Configure()
{
  // LyotropicWithDivision::Configure is Lyotropic::Configure; the conserve_phi
  // correction is switched on below, against the relaxed total
  LyotropicGPU::Configure();
  RelaxFreeEnergy();
  ResetHydrodynamics();
  ConfigurePhenotype();
  if(conserve_phi)
  {
    const int r = mass_lb_set_phi_conservation(lattice, 1, totalphi);
    if(r != MASS_LB_OK)
      throw error_msg(mass_gpu::abi_error("mass_lb_set_phi_conservation", r));
  }
}

void GoOrGrowGPU::RelaxFreeEnergy()
{
  if(relax_steps == 0 || (!relax_phi && !relax_Q))
    return;
  double relaxed_phi = 0.;
  const int r = mass_lb_relax_free_energy(lattice, relax_steps, relax_dt, relax_phi, relax_Q,
                                          &relaxed_phi);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_relax_free_energy", r));
  totalphi = relaxed_phi;
  ptot = relaxed_phi;
}

void GoOrGrowGPU::ResetHydrodynamics()
{
  // every population at the rest equilibrium, ftot summed site by site
  double ftotal = 0.;
  const auto fe = mass_gpu::equilibrium(0., 0., rho);
  for(unsigned k = 0; k < DomainSize; ++k)
  {
    ff[k] = fe;
    for(double f : fe) ftotal += f;
  }
  ftot = ftotal;
  std::vector<double> flat;
  mass_gpu::flatten(ff, flat);
  const int r = mass_lb_upload_field(lattice, MASS_LB_FF, flat.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_upload_field", r));
}

double GoOrGrowGPU::HostLaplacian(const std::vector<double>& a, unsigned k) const
{
  // Periodic axes wrap. A wall's ghost holds the Neumann copy of the domain
  // site next to it (ApplyNeumann / ApplyNeumannChannel), which for the
  // five-point stencil is the site itself. Channels (bc 1, 2) have walls at
  // y = 0 and y = LY-1, boxes (bc 3, 4) on all four sides; every other bc
  // is periodic.
  const unsigned x = GetXPosition(k), y = k % LY;
  const bool xwall = BC == 3 || BC == 4;
  const bool ywall = BC >= 1 && BC <= 4;
  auto at = [&](unsigned xx, unsigned yy) { return a[yy + LY*xx]; };
  const unsigned xp = x + 1 == LX ? (xwall ? x : 0) : x + 1;
  const unsigned xm = x == 0 ? (xwall ? x : LX - 1) : x - 1;
  const unsigned yp = y + 1 == LY ? (ywall ? y : 0) : y + 1;
  const unsigned ym = y == 0 ? (ywall ? y : LY - 1) : y - 1;
  // src/lb.hpp:129-136, neighbours in D2Q9 order +x, -x, +y, -y
  return at(xp, y) + at(xm, y) + at(x, yp) + at(x, ym) - 4*a[k] + 0*(1/12.);
}

void GoOrGrowGPU::ConfigurePhenotype()
{
  // phi after the relaxation
  int r = mass_lb_download(lattice, MASS_LB_PHI, phi.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_download", r));

  if(chi_config == "noise")
  {
    for(unsigned k = 0; k < DomainSize; ++k)
      chi[k] = random_normal();

    constexpr double smooth_rate = 0.2;
    const unsigned smooth_steps =
      chi_length > 0 ? static_cast<unsigned>(ceil(chi_length*chi_length/(2*smooth_rate))) : 0u;
    std::vector<double> next(DomainSize);
    for(unsigned s = 0; s < smooth_steps; ++s)
    {
      for(unsigned k = 0; k < DomainSize; ++k)
        next[k] = chi[k] + smooth_rate*HostLaplacian(chi, k);
      swap(chi, next);
    }

    double mean = 0.;
    for(unsigned k = 0; k < DomainSize; ++k)
      mean += chi[k];
    mean /= DomainSize;

    double variance = 0.;
    for(unsigned k = 0; k < DomainSize; ++k)
    {
      chi[k] -= mean;
      variance += chi[k]*chi[k];
    }
    variance /= DomainSize;

    const double amplitude = sqrt(chi_noise);
    const double norm = variance > 0 ? amplitude/sqrt(variance) : 0.;
    for(unsigned k = 0; k < DomainSize; ++k)
      chi[k] = chi0 + norm*chi[k];
  }
  else if(chi_config == "front")
  {
    const double length = chi_length > 0 ? chi_length : 1.;
    const double center = .5*(LX - 1);
    for(unsigned k = 0; k < DomainSize; ++k)
    {
      const double x = GetXPosition(k);
      chi[k] = .5*(1. - tanh((x - center)/length));
    }
  }
  else
    throw error_msg("error: chi configuration '", chi_config, "' unknown.");

  // m = phi*chi projected onto [0, max(phi, 0)] (ProjectM, :218-228); the
  // device derives chi = m/phi from it (UpdatePhenotypeQuantities)
  for(unsigned k = 0; k < DomainSize; ++k)
  {
    double v = phi[k]*chi[k];
    const double upper = phi[k] > 0 ? phi[k] : 0.;
    if(v < 0) v = 0;
    else if(v > upper) v = upper;
    m[k] = v;
  }
  r = mass_lb_upload_field(lattice, MASS_LB_M, m.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_upload_field", r));
}

void GoOrGrowGPU::SyncPhenotype()
{
  int r = mass_lb_download(lattice, MASS_LB_M, m.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_download", r));
  r = mass_lb_download(lattice, MASS_LB_CHI, chi.data());
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_download", r));
}

option_list GoOrGrowGPU::GetOptions()
{
  auto options = LyotropicWithDivisionGPU::GetOptions();
  options[0].add_options()
    ("B", opt::value<double>(&B),
     "crowding/compressibility penalty strength")
    ("Snem", opt::value<double>(&Snem),
     "preferred value of one half Tr(Q^2)")
    ("Dchi", opt::value<double>(&Dchi),
     "phenotype diffusion coefficient")
    ("Achi", opt::value<double>(&Achi),
     "phenotype switching double-well barrier")
    ("Ochi", opt::value<double>(&Ochi),
     "phenotype switching bias strength")
    ("phiswitch", opt::value<double>(&phiswitch),
     "phi threshold for phenotype switching bias")
    ("growTogether", opt::value<int>(&growTogether),
     "m growth source: 0 uses R, 1 uses chi*R")
    ("chi-config", opt::value<string>(&chi_config),
     "phenotype initialization mode: noise or front")
    ("chi0", opt::value<double>(&chi0),
     "initial phenotype mean")
    ("chi-noise", opt::value<double>(&chi_noise),
     "initial phenotype variance")
    ("chi-length", opt::value<double>(&chi_length),
     "initial phenotype correlation length")
    ("relax-steps", opt::value<unsigned>(&relax_steps),
     "dry free-energy relaxation steps before official dynamics")
    ("relax-dt", opt::value<double>(&relax_dt),
     "time step multiplier for dry free-energy relaxation")
    ("relax-phi", opt::value<int>(&relax_phi),
     "relax phi by Cahn-Hilliard free-energy descent before official dynamics")
    ("relax-Q", opt::value<int>(&relax_Q),
     "relax Q by molecular-field free-energy descent before official dynamics");
  return options;
}
