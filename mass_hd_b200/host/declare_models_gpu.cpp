// Model registrations of the standalone GPU build. Inside the reference tree
// the same declare_model calls go into src/declare_models.cpp; here the
// reference's names ("lyotropic", "lyotropic-with-division", "go-or-grow",
// "nematic") are registered as well, so unchanged reference runcards run on
// the GPU.
#include "models.hpp"
#include "lyotropic_gpu.hpp"
#include "lyotropic_with_division_gpu.hpp"
#include "go_or_grow_gpu.hpp"
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
  const char* gog = "Go-or-grow lyotropic model with a passive phenotype field chi, with its "
                    "time step on a B200 GPU.";
  declare_model<GoOrGrowGPU>("go-or-grow-gpu", gog);
  declare_model<LyotropicGPU>("lyotropic", lyo);
  declare_model<LyotropicWithDivisionGPU>("lyotropic-with-division", div);
  declare_model<GoOrGrowGPU>("go-or-grow", gog);
  declare_model<NematicGPU>("nematic", nem);
}
