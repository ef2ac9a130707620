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
  // the reference's schedule (:37, :73): a mask is redrawn when its counter
  // runs out, then the counter restarts from its life time
  int kinds = 0;
  if(not division_count--)
  {
    kinds |= 1;
    division_count = division_time;
  }
  if(not death_count--)
  {
    kinds |= 2;
    death_count = death_time;
  }
  if(!kinds) return;
  // The device takes one uniform per site with phi >= .5 and mask, in site
  // order, from a queue of the reference generator's values. 2*LX*LY of
  // them cover one draw of both masks of any count. The host learns how many
  // were consumed from the draws the device has finished, without waiting,
  // and keeps 2*LX*LY more for each draw still in flight and the next one,
  // so it runs up to three draws ahead of the device.
  long long consumed = 0;
  int pending = 0;
  int r = mass_lb_mask_progress(lattice, &consumed, &pending);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_mask_progress", r));
  if(pending > 2)
  {
    r = mass_lb_mask_consumed(lattice, &consumed);
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_mask_consumed", r));
    pending = 0;
  }
  const long long want = consumed + 2*static_cast<long long>(DomainSize)*(pending + 1);
  if(supplied < want)
  {
    const size_t n = static_cast<size_t>(want - supplied);
    // the draws are written straight into the library's pinned staging
    double* u = nullptr;
    r = mass_lb_mask_staging(lattice, static_cast<long long>(n), &u);
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_mask_staging", r));
#ifdef MASS_GPU_STANDALONE
    random_reals(u, n);   // the same values as n random_real() calls
#else
    for(size_t i = 0; i < n; ++i) u[i] = random_real();
#endif
    r = mass_lb_mask_supply(lattice, u, static_cast<long long>(n));
    if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_mask_supply", r));
    supplied = want;
  }
  r = mass_lb_draw_masks_queued(lattice, kinds, division_rate, division_radius, death_rate,
                                death_radius, phi_critical, alpha, beta);
  if(r != MASS_LB_OK) throw error_msg(mass_gpu::abi_error("mass_lb_draw_masks_queued", r));
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

void LyotropicWithDivisionGPU::Step()
{
  // Step() must not throw (src/models.hpp:81-86): a failure is kept and
  // reported by the next RuntimeChecks().
  if(!step_error.empty()) return;
  try { SetMasks(); }
  catch(const error_msg& e) { step_error = e.what(); return; }
  LyotropicGPU::Step();
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
