#include "header.hpp"
#include "lyotropic_with_division_gpu.hpp"
#include "error_msg.hpp"
#include "random.hpp"
#include "mass_lb_ext.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>

using namespace std;
namespace opt = boost::program_options;

LyotropicWithDivisionGPU::LyotropicWithDivisionGPU(unsigned LX_, unsigned LY_, unsigned BC_)
  : LyotropicGPU(LX_, LY_, BC_)
{}

void LyotropicWithDivisionGPU::Initialize()
{
  LyotropicGPU::Initialize();
  division_mask.assign(DomainSize, false);
  death_mask.assign(DomainSize, false);
  division_count = death_count = 0u;
  // as src/models/lyotropic-with-division.cpp:29-30
  conserve_phi = ((alpha == 0 || division_rate == 0) && (beta == 0 || death_rate == 0));
}

void LyotropicWithDivisionGPU::Configure()
{
  LyotropicGPU::Configure();
  if(conserve_phi)
  {
    const int r = mass_lb_set_phi_conservation(lattice, 1, totalphi);
    if(r != MASS_LB_OK)
      throw error_msg(mass_gpu::abi_error("mass_lb_set_phi_conservation", r),
                      " (division and death are off, so phi is conserved by a lattice-wide "
                      "correction; run with precision=fp64)");
  }
}

void LyotropicWithDivisionGPU::SetMasks()
{
  long long candidates = -1;
  auto draw = [&](int kind, double rate_coef, double radius) {
    if(candidates < 0)
    {
      const int r = mass_lb_mask_candidates(lattice, &candidates);
      if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_mask_candidates", r));
    }
    // one random_real() per site with phi >= .5, in site order, from the
    // reference's generator; the centres and circles are drawn on the device
    last_candidates = candidates;
    const double* draws = TakeDraws(static_cast<size_t>(candidates));
    const int r = mass_lb_draw_mask(lattice, kind, draws, candidates, rate_coef,
                                    phi_critical, radius, alpha, beta);
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_draw_mask", r));
  };
  if(not division_count--)
  {
    draw(0, division_rate, division_radius);
    division_count = division_time;
  }
  if(not death_count--)
  {
    draw(1, death_rate, death_radius);
    death_count = death_time;
  }
}

void LyotropicWithDivisionGPU::SyncMasks()
{
  std::vector<unsigned char> bytes(DomainSize);
  std::vector<bool>* masks[2] = {&division_mask, &death_mask};
  for(int kind = 0; kind < 2; ++kind)
  {
    const int r = mass_lb_get_mask(lattice, kind, bytes.data());
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_get_mask", r));
    for(unsigned k = 0; k < DomainSize; ++k) (*masks[kind])[k] = bytes[k] != 0;
  }
}

void LyotropicWithDivisionGPU::DrawAhead(size_t n)
{
  if(fifo.size() - fifo_head >= n) return;
  if(fifo_head > 0)
  {
    fifo.erase(fifo.begin(), fifo.begin() + static_cast<std::ptrdiff_t>(fifo_head));
    fifo_head = 0;
  }
  const size_t have = fifo.size();
  fifo.resize(n);
#ifdef MASS_GPU_STANDALONE
  random_reals(fifo.data() + have, n - have);   // the same values, in bulk
#else
  for(size_t i = have; i < n; ++i) fifo[i] = random_real();
#endif
}

const double* LyotropicWithDivisionGPU::TakeDraws(size_t n)
{
  DrawAhead(n);
  const double* p = fifo.data() + fifo_head;
  fifo_head += n;
  return p;
}

void LyotropicWithDivisionGPU::Step()
{
  // Step() must not throw (src/models.hpp:81-86): a failure is kept and
  // reported by the next RuntimeChecks().
  if(!step_error.empty()) return;
  try { SetMasks(); }
  catch(const error_msg& e) { step_error = e.what(); return; }
  LyotropicGPU::Step();
  // while the device steps, draw the values of the next masks (two masks
  // of about the last candidate count); only masks consume the generator
  // after Configure(), so drawing early leaves every value in its place
  DrawAhead(2*static_cast<size_t>(last_candidates));
}

void LyotropicWithDivisionGPU::RuntimeChecks()
{
  LyotropicGPU::RuntimeChecks();
  // phi is checked only when it is conserved (src/models/lyotropic.cpp:538-548)
  if(conserve_phi)
  {
    double fcheck = 0, pcheck = 0;
    int bad = 0;
    const int r = mass_lb_checks(lattice, &fcheck, &pcheck, &bad);
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_checks", r));
    if(abs(ptot - pcheck) > 1)
      throw error_msg("phi is not conserved (", ptot, "/", pcheck, ")");
  }
}

option_list LyotropicWithDivisionGPU::GetOptions()
{
  auto options = LyotropicGPU::GetOptions();
  options[0].add_options()
    ("alpha", opt::value<double>(&alpha), "division strength")
    ("beta", opt::value<double>(&beta), "death strength")
    ("division-rate", opt::value<double>(&division_rate), "division rate")
    ("division-time", opt::value<double>(&division_time), "division life time")
    ("division-radius", opt::value<double>(&division_radius), "division radius")
    ("death-rate", opt::value<double>(&death_rate), "death rate")
    ("death-time", opt::value<double>(&death_time), "death life time")
    ("death-radius", opt::value<double>(&death_radius), "death radius")
    ("phi-critical", opt::value<double>(&phi_critical), "phi critical");
  return options;
}
