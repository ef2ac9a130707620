// Model registrations of the standalone GPU build. Inside the reference tree
// the same two declare_model calls go into src/declare_models.cpp (see
// INTEGRATION.md); here the reference's names "lyotropic" and "nematic" are
// registered as well, so unchanged reference runcards run on the GPU.
#include "models.hpp"
#include "lyotropic_gpu.hpp"
#include "lyotropic_with_division_gpu.hpp"
#include "nematic_gpu.hpp"

void DeclareModels()
{
  static bool done = false;
  if(done) return;
  done = true;
  const char* lyo = "Biphasic, lyotropic, nematic model (10.1103/PhysRevLett.113.248303) "
                    "with its time step on a B200 GPU.";
  const char* nem = "Active nematic model with its time step on a B200 GPU.";
  declare_model<LyotropicGPU>("lyotropic-gpu", lyo);
  declare_model<NematicGPU>("nematic-gpu", nem);
  const char* div = "Lyotropic model with cell division and death, with its time step on a "
                    "B200 GPU.";
  declare_model<LyotropicWithDivisionGPU>("lyotropic-with-division-gpu", div);
  declare_model<LyotropicGPU>("lyotropic", lyo);
  declare_model<LyotropicWithDivisionGPU>("lyotropic-with-division", div);
  declare_model<NematicGPU>("nematic", nem);
}
