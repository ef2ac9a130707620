// Oracle harness around the reference's OWN model translation units.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the
// reference sources (src/geometry.cpp, src/random.cpp, src/serialization.cpp,
// src/models/lyotropic.cpp, src/models/nematic.cpp,
// src/models/lyotropic-with-division.cpp, src/models/go-or-grow.cpp) by
// oracle/Makefile into
// oracle/_ref/libmass_ref.so. Nothing in the product links it; the tests,
// the golden-fixture generator and bench.py's reference arm load it through
// ctypes as the checker / CPU baseline.
//
// It replaces the pieces of the reference driver that those TUs need:
//   * Model::Model            (src/models.cpp:16)
//   * globals nthreads, nsubsteps, time_step (src/main.cpp, used extern in
//     src/models/lyotropic.cpp:12-13)
//   * WriteParams()/WriteFrame() bodies (src/write.cpp:28-106), restated so
//     that JSON can be produced for a given path without the global driver.
// and exposes a C ABI to set options by runcard name, seed and configure,
// overwrite the primary state, step, and read any field back in memory.

#include "header.hpp"
#include "models.hpp"
#include "models/lyotropic.hpp"
#include "models/lyotropic-with-division.hpp"
#include "models/go-or-grow.hpp"
#include "models/nematic.hpp"
#include "random.hpp"
#include "serialization.hpp"
#include "error_msg.hpp"

#include <cstring>
#include <fstream>
#include <chrono>

unsigned nthreads = 0, nsubsteps = 1;
double time_step = 1.;

Model::Model(unsigned LX, unsigned LY, unsigned BC, GridType Type)
  : Grid(LX, LY, Type), BC(BC)
{}

namespace {

// Common interface over the two reference models (they share no base beyond
// Model, and their fields are protected, so each gets an access subclass).
struct RefModel
{
  virtual ~RefModel() {}
  virtual Model& model() = 0;
  virtual option_list options() = 0;
  virtual ScalarField* scalar(const std::string&) = 0;
  virtual LBField* lb(const std::string&) = 0;
  virtual void reset_totals() = 0;
  virtual void write_params(std::ostream&, unsigned nsteps, unsigned ninfo,
                            unsigned nstart, const std::string&) = 0;
  virtual void write_frame(std::ostream&) = 0;
  virtual unsigned lx() = 0;
  virtual unsigned ly() = 0;
  virtual unsigned bc() = 0;
  // boolean masks of the division models (null elsewhere)
  virtual const std::vector<bool>* mask(const std::string&) { return nullptr; }
  // scalar members (totalphi, countphi, conserve_phi); false if absent
  virtual bool value(const std::string&, double*) { return false; }
  option_list opts;
};

template<class Archive, class M>
void write_params_common(Archive& ar, M& m, unsigned LX, unsigned LY,
                         unsigned BC, unsigned nsteps, unsigned ninfo,
                         unsigned nstart, std::string model_name)
{
  // same keys, same order as src/write.cpp:75-84
  unsigned nsubsteps_ = ::nsubsteps;
  unsigned& nsubsteps = nsubsteps_;
  ar & auto_name(LX)
     & auto_name(LY)
     & auto_name(BC)
     & auto_name(nsteps)
     & auto_name(nsubsteps)
     & auto_name(ninfo)
     & auto_name(nstart)
     & auto_name(model_name);
  m.serialize_params(ar);
}

// Lyotropic and the models derived from it share fields and serialization.
template<class Base>
struct LyoAccessT : Base, RefModel
{
  LyoAccessT(unsigned LX, unsigned LY, unsigned BC) : Base(LX, LY, BC) {}
  Model& model() override { return *this; }
  option_list options() override { return Base::GetOptions(); }
  unsigned lx() override { return this->LX; }
  unsigned ly() override { return this->LY; }
  unsigned bc() override { return this->BC; }
  bool value(const std::string& name, double* out) override
  {
    if(name=="totalphi") { *out = this->totalphi; return true; }
    if(name=="countphi") { *out = this->countphi; return true; }
    if(name=="conserve_phi") { *out = this->conserve_phi ? 1. : 0.; return true; }
    return false;
  }
  ScalarField* scalar(const std::string& name) override
  {
#define F(x) if(name==#x) return &this->x;
    F(QQxx) F(QQyx) F(QNxx) F(QNyx) F(phi) F(phn) F(phi_tmp) F(n) F(ux) F(uy)
    F(ux_phi) F(uy_phi) F(HHxx) F(HHyx) F(MU) F(dxQQxx) F(dyQQxx) F(dxQQyx)
    F(dyQQyx) F(sigmaXX) F(sigmaYY) F(sigmaYX) F(sigmaXY) F(sigma_bulk)
    F(sigma_elastic_xx) F(sigma_elastic_yx) F(sigma_phase_field_xx)
    F(sigma_phase_field_yx) F(sigma_active_xx) F(sigma_active_yx)
#undef F
    return nullptr;
  }
  LBField* lb(const std::string& name) override
  {
    if(name=="ff") return &this->ff;
    if(name=="fn") return &this->fn;
    return nullptr;
  }
  void reset_totals() override
  {
    this->ftot = 0; this->ptot = 0;
    for(unsigned k=0; k<this->DomainSize; ++k)
    {
      for(unsigned v=0; v<lbq; ++v) this->ftot += this->ff[k][v];
      this->ptot += this->phi[k];
    }
  }
  void write_params(std::ostream& os, unsigned nsteps, unsigned ninfo,
                    unsigned nstart, const std::string& name) override
  {
    oarchive ar(os, "parameters", 1);
    write_params_common(ar, *this, this->LX, this->LY, this->BC, nsteps, ninfo, nstart, name);
    if(ar.bad_value()) throw error_msg("nan found while writing file.");
  }
  void write_frame(std::ostream& os) override
  {
    oarchive ar(os, "frame", 1);
    this->serialize_frame(ar);
    if(ar.bad_value()) throw error_msg("nan found while writing file.");
  }
};

using LyoAccess = LyoAccessT<Lyotropic>;

// LyotropicWithDivision (src/models/lyotropic-with-division.cpp) with its
// division / death masks readable
struct DivAccess : LyoAccessT<LyotropicWithDivision>
{
  DivAccess(unsigned LX, unsigned LY, unsigned BC) : LyoAccessT(LX, LY, BC) {}
  const std::vector<bool>* mask(const std::string& name) override
  {
    if(name=="division_mask") return &division_mask;
    if(name=="death_mask") return &death_mask;
    return nullptr;
  }
};

// GoOrGrow (src/models/go-or-grow.cpp): the division masks plus the
// phenotype fields m, mN, m_tmp, chi
struct GogAccess : LyoAccessT<GoOrGrow>
{
  GogAccess(unsigned LX, unsigned LY, unsigned BC) : LyoAccessT(LX, LY, BC) {}
  const std::vector<bool>* mask(const std::string& name) override
  {
    if(name=="division_mask") return &division_mask;
    if(name=="death_mask") return &death_mask;
    return nullptr;
  }
  ScalarField* scalar(const std::string& name) override
  {
    if(name=="m") return &m;
    if(name=="mN") return &mN;
    if(name=="m_tmp") return &m_tmp;
    if(name=="chi") return &chi;
    return LyoAccessT::scalar(name);
  }
};

struct NemAccess : Nematic, RefModel
{
  NemAccess(unsigned LX, unsigned LY, unsigned BC) : Nematic(LX, LY, BC) {}
  Model& model() override { return *this; }
  option_list options() override { return Nematic::GetOptions(); }
  unsigned lx() override { return LX; }
  unsigned ly() override { return LY; }
  unsigned bc() override { return BC; }
  ScalarField* scalar(const std::string& name) override
  {
#define F(x) if(name==#x) return &x;
    F(QQxx) F(QQyx) F(QNxx) F(QNyx) F(n) F(ux) F(uy) F(HHxx) F(HHyx)
    F(dxQQxx) F(dyQQxx) F(dxQQyx) F(dyQQyx) F(sigmaXX) F(sigmaYY) F(sigmaYX)
    F(sigmaXY)
#undef F
    return nullptr;
  }
  LBField* lb(const std::string& name) override
  {
    if(name=="ff") return &ff;
    if(name=="fn") return &fn;
    return nullptr;
  }
  void reset_totals() override
  {
    ftot = 0;
    for(unsigned k=0; k<DomainSize; ++k)
      for(unsigned v=0; v<lbq; ++v) ftot += ff[k][v];
  }
  void write_params(std::ostream& os, unsigned nsteps, unsigned ninfo,
                    unsigned nstart, const std::string& name) override
  {
    oarchive ar(os, "parameters", 1);
    write_params_common(ar, *this, LX, LY, BC, nsteps, ninfo, nstart, name);
    if(ar.bad_value()) throw error_msg("nan found while writing file.");
  }
  void write_frame(std::ostream& os) override
  {
    oarchive ar(os, "frame", 1);
    serialize_frame(ar);
    if(ar.bad_value()) throw error_msg("nan found while writing file.");
  }
};

thread_local std::string last_error;

} // namespace

extern "C" {

/** Last error message of this thread (empty if none). */
const char* ref_last_error() { return last_error.c_str(); }

/** Construct "lyotropic", "lyotropic-with-division", "go-or-grow" or
 * "nematic" with the
 * factory arguments of
 * declare_model (src/models.hpp:197-205): (LX, LY, BC). */
void* ref_new(const char* model, unsigned LX, unsigned LY, unsigned BC)
{
  try {
    RefModel* m = nullptr;
    if(std::strcmp(model, "lyotropic")==0) m = new LyoAccess(LX, LY, BC);
    else if(std::strcmp(model, "lyotropic-with-division")==0) m = new DivAccess(LX, LY, BC);
    else if(std::strcmp(model, "go-or-grow")==0) m = new GogAccess(LX, LY, BC);
    else if(std::strcmp(model, "nematic")==0) m = new NemAccess(LX, LY, BC);
    else { last_error = "unknown model"; return nullptr; }
    m->opts = m->options();
    return m;
  } catch(const std::exception& e) { last_error = e.what(); return nullptr; }
}

void ref_free(void* h) { delete static_cast<RefModel*>(h); }

/** Assign a runcard option by name (GetOptions names). 0 ok, -1 unknown,
 * -2 unparsable. */
int ref_set_option(void* h, const char* name, const char* value)
{
  auto* m = static_cast<RefModel*>(h);
  for(const auto& d : m->opts)
  {
    const int r = d.set_option(name, value);
    if(r != -1) return r;
  }
  return -1;
}

/** Model::Initialize() (allocation, derived params). */
int ref_initialize(void* h)
{
  try { static_cast<RefModel*>(h)->model().Initialize(); return 0; }
  catch(const error_msg& e) { last_error = e.what(); return -1; }
  catch(const std::exception& e) { last_error = e.what(); return -1; }
}

/** set_seed(seed) then Model::Configure() (src/options.cpp:151, main.cpp:251). */
int ref_configure(void* h, unsigned seed)
{
  try {
    set_seed(seed);
    static_cast<RefModel*>(h)->model().Configure();
    return 0;
  }
  catch(const error_msg& e) { last_error = e.what(); return -1; }
  catch(const std::exception& e) { last_error = e.what(); return -1; }
}

/** Overwrite domain values of one field. For "ff"/"fn" `src` holds
 * DomainSize*9 doubles, site-major ([k][v]); otherwise DomainSize doubles. */
int ref_set_field(void* h, const char* name, const double* src)
{
  auto* m = static_cast<RefModel*>(h);
  const unsigned N = m->lx()*m->ly();
  if(LBField* f = m->lb(name))
  {
    for(unsigned k=0; k<N; ++k)
      for(unsigned v=0; v<lbq; ++v) (*f)[k][v] = src[9*k+v];
    return 0;
  }
  if(ScalarField* f = m->scalar(name))
  {
    for(unsigned k=0; k<N; ++k) (*f)[k] = src[k];
    return 0;
  }
  last_error = std::string("unknown field ") + name;
  return -1;
}

/** Copy domain values of one field out (same layout as ref_set_field). */
int ref_get_field(void* h, const char* name, double* dst)
{
  auto* m = static_cast<RefModel*>(h);
  const unsigned N = m->lx()*m->ly();
  if(LBField* f = m->lb(name))
  {
    for(unsigned k=0; k<N; ++k)
      for(unsigned v=0; v<lbq; ++v) dst[9*k+v] = (*f)[k][v];
    return 0;
  }
  if(ScalarField* f = m->scalar(name))
  {
    for(unsigned k=0; k<N; ++k) dst[k] = (*f)[k];
    return 0;
  }
  last_error = std::string("unknown field ") + name;
  return -1;
}

/** Copy a boolean mask of the division models (division_mask,
 * death_mask) out as 0/1 bytes in site order. */
int ref_get_mask(void* h, const char* name, unsigned char* dst)
{
  auto* m = static_cast<RefModel*>(h);
  const std::vector<bool>* v = m->mask(name);
  if(!v) { last_error = std::string("unknown mask ") + name; return -1; }
  for(size_t k=0; k<v->size(); ++k) dst[k] = (*v)[k] ? 1 : 0;
  return 0;
}

/** A scalar member of the lyotropic models: totalphi, countphi,
 * conserve_phi (1 or 0). */
int ref_get_value(void* h, const char* name, double* out)
{
  auto* m = static_cast<RefModel*>(h);
  if(!m->value(name, out)) { last_error = std::string("unknown value ") + name; return -1; }
  return 0;
}

/** Recompute the conservation totals (ftot, ptot) from the current state,
 * as Configure() does (src/models/lyotropic.cpp:158-159). */
void ref_reset_totals(void* h) { static_cast<RefModel*>(h)->reset_totals(); }

/** Run `n` calls of Model::Step() with `threads` OpenMP threads
 * (0 = serial, the `-t0` default, src/options.cpp:51-54). */
int ref_step(void* h, unsigned n, unsigned threads)
{
  nthreads = threads;
  auto& mod = static_cast<RefModel*>(h)->model();
  for(unsigned i=0; i<n; ++i) mod.Step();
  return 0;
}

/** Wall time in seconds of `n` Step() calls with `threads` threads. */
double ref_time_steps(void* h, unsigned n, unsigned threads)
{
  nthreads = threads;
  auto& mod = static_cast<RefModel*>(h)->model();
  const auto t0 = std::chrono::steady_clock::now();
  for(unsigned i=0; i<n; ++i) mod.Step();
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

/** Model::RuntimeChecks(); 0 ok, -1 error_msg thrown (message in
 * ref_last_error). */
int ref_runtime_checks(void* h)
{
  try { static_cast<RefModel*>(h)->model().RuntimeChecks(); return 0; }
  catch(const error_msg& e) { last_error = e.what(); return -1; }
  catch(const warning_msg& e) { last_error = e.what(); return -2; }
}

/** parameters.json as WriteParams() would write it (src/write.cpp:63-91). */
int ref_write_params(void* h, const char* path, unsigned nsteps,
                     unsigned ninfo, unsigned nstart, const char* model_name)
{
  try {
    std::stringstream buffer;
    static_cast<RefModel*>(h)->write_params(buffer, nsteps, ninfo, nstart,
                                            model_name);
    std::ofstream ofs(path, std::ios::out);
    ofs << buffer.rdbuf();
    return 0;
  } catch(const std::exception& e) { last_error = e.what(); return -1; }
  catch(const error_msg& e) { last_error = e.what(); return -1; }
}

/** frame<t>.json body as WriteFrame() would write it (src/write.cpp:28-46). */
int ref_write_frame(void* h, const char* path)
{
  try {
    std::stringstream buffer;
    static_cast<RefModel*>(h)->write_frame(buffer);
    std::ofstream ofs(path, std::ios::out);
    ofs << buffer.rdbuf();
    return 0;
  } catch(const std::exception& e) { last_error = e.what(); return -1; }
  catch(const error_msg& e) { last_error = e.what(); return -1; }
}

/** random_real() draws from the reference's global generator
 * (src/random.cpp:21), after set_seed(seed) when seed_first != 0. */
void ref_random_reals(unsigned seed, int seed_first, unsigned n, double* out)
{
  if(seed_first) set_seed(seed);
  for(unsigned i=0; i<n; ++i) out[i] = random_real();
}

} // extern "C"
