// Writes frame JSON with the standalone plugin build's archive
// (mass_hd_b200/host/compat/serialization.hpp) from raw little-endian double
// files <dir>/<field>.bin, for the field lists of the lyotropic and nematic
// frames (member names and order of serialize_frame).
//   write_frame lyo|nem <dir> <out.json>
#include "serialization.hpp"

#include <array>
#include <cstring>
#include <iterator>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

static std::vector<double> load(const std::string& path)
{
  std::ifstream in(path, std::ios::binary);
  std::vector<char> raw((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  std::vector<double> v(raw.size()/sizeof(double));
  std::memcpy(v.data(), raw.data(), v.size()*sizeof(double));
  return v;
}

int main(int argc, char** argv)
{
  if(argc < 4) return 2;
  const std::string kind = argv[1], dir = argv[2];
  const std::vector<double> flat = load(dir + "/ff.bin");
  std::vector<std::array<double, 9>> ff(flat.size()/9);
  for(size_t k = 0; k < ff.size(); ++k)
    for(int v = 0; v < 9; ++v) ff[k][v] = flat[9*k + v];
  std::vector<double> QQxx = load(dir + "/QQxx.bin"), QQyx = load(dir + "/QQyx.bin");
  std::ofstream os(argv[3]);
  oarchive ar(os, "frame", 1);
  ar & auto_name(ff) & auto_name(QQxx) & auto_name(QQyx);
  if(kind == "lyo")
  {
    std::vector<double> phi = load(dir + "/phi.bin"), sigmaXX = load(dir + "/sigmaXX.bin"),
      sigmaXY = load(dir + "/sigmaXY.bin"), sigmaYX = load(dir + "/sigmaYX.bin"),
      sigmaYY = load(dir + "/sigmaYY.bin"), sigma_bulk = load(dir + "/sigma_bulk.bin"),
      sigma_elastic_xx = load(dir + "/sigma_elastic_xx.bin"),
      sigma_elastic_yx = load(dir + "/sigma_elastic_yx.bin"),
      sigma_phase_field_xx = load(dir + "/sigma_phase_field_xx.bin"),
      sigma_phase_field_yx = load(dir + "/sigma_phase_field_yx.bin"),
      sigma_active_xx = load(dir + "/sigma_active_xx.bin"),
      sigma_active_yx = load(dir + "/sigma_active_yx.bin");
    ar & auto_name(phi) & auto_name(sigmaXX) & auto_name(sigmaXY) & auto_name(sigmaYX)
       & auto_name(sigmaYY) & auto_name(sigma_bulk) & auto_name(sigma_elastic_xx)
       & auto_name(sigma_elastic_yx) & auto_name(sigma_phase_field_xx)
       & auto_name(sigma_phase_field_yx) & auto_name(sigma_active_xx)
       & auto_name(sigma_active_yx);
  }
  return 0;
}
