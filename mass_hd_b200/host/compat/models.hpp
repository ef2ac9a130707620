// The model plugin interface of MASS, restated for the standalone build of
// the GPU plugin: the Grid members models read (LX, LY, Type, DomainSize,
// TotalSize, site indexing k = y + LY*x; reference src/geometry.hpp:334-431),
// the abstract Model with its virtual life cycle (src/models.hpp:30-116),
// the type-erased serializer pointer ModelPtr (src/models.hpp:129-187) and
// the name registry declare_model / NewModel (src/models.hpp:189-214,
// src/models.cpp:32-49). Inside the reference tree the reference's own
// models.hpp is used instead.
#ifndef MASS_GPU_COMPAT_MODELS_HPP_
#define MASS_GPU_COMPAT_MODELS_HPP_

#include "header.hpp"
#include "serialization.hpp"

#include <functional>
#include <string>
#include <vector>

using option_list = std::vector<boost::program_options::options_description>;

class Grid
{
public:
  enum class GridType { Periodic = 0, Layer = 1 };

protected:
  unsigned LX = 0, LY = 0;
  GridType Type = GridType::Periodic;
  unsigned DomainSize = 0;
  unsigned TotalSize = 0;

public:
  Grid() = default;
  Grid(unsigned LX_, unsigned LY_, GridType Type_) { SetSize(LX_, LY_, Type_); }
  virtual ~Grid() {}
  void SetSize(unsigned LX_, unsigned LY_, GridType Type_)
  {
    LX = LX_; LY = LY_; Type = Type_;
    DomainSize = LX*LY;
    TotalSize = Type == GridType::Periodic ? DomainSize : (LX + 2)*(LY + 2);
  }
  unsigned GetXPosition(unsigned k) const { return k/LY; }
  unsigned GetYPosition(unsigned k) const { return k%LY; }
  unsigned GetDomainIndex(unsigned x, unsigned y) const { return y + LY*x; }
  unsigned GetSize() const { return DomainSize; }
};

class Model : public Grid
{
protected:
  unsigned BC = 0;

public:
  Model() = default;
  Model(unsigned LX_, unsigned LY_, unsigned BC_, GridType Type_)
    : Grid(LX_, LY_, Type_), BC(BC_) {}
  virtual ~Model() {}
  virtual void Initialize() = 0;
  virtual void Configure() = 0;
  virtual option_list GetOptions() = 0;
  virtual void Pre() {}
  virtual void Step() = 0;
  virtual void Post() {}
  virtual void RuntimeChecks() {}
  virtual void RuntimeStats() {}
  virtual void PreRunStats() {}
};

struct ModelPtr
{
  struct SerializerPtr
  {
    Model* ptr;
    explicit SerializerPtr(Model* p) : ptr(p) {}
    virtual ~SerializerPtr() {}
    virtual void serialize_params(oarchive&) = 0;
    virtual void serialize_params(iarchive&) = 0;
    virtual void serialize_frame(oarchive&) = 0;
    virtual void serialize_frame(iarchive&) = 0;
  };

  template<class Derived>
  struct SerializerPtr_tmpl : SerializerPtr
  {
    explicit SerializerPtr_tmpl(Derived* p) : SerializerPtr(p) {}
    void serialize_params(oarchive& ar) override { static_cast<Derived*>(ptr)->serialize_params(ar); }
    void serialize_params(iarchive& ar) override { static_cast<Derived*>(ptr)->serialize_params(ar); }
    void serialize_frame(oarchive& ar) override { static_cast<Derived*>(ptr)->serialize_frame(ar); }
    void serialize_frame(iarchive& ar) override { static_cast<Derived*>(ptr)->serialize_frame(ar); }
  };

  SerializerPtr* ptr = nullptr;
  ModelPtr() = default;
  template<class Derived>
  explicit ModelPtr(Derived* m) : ptr(new SerializerPtr_tmpl<Derived>(m)) {}
  Model* operator->() { return ptr->ptr; }
  const Model* operator->() const { return ptr->ptr; }
};

using Factory = std::function<ModelPtr(unsigned, unsigned, unsigned)>;

void _add_model(std::string name, std::string desc, Factory fact);

template<class T>
void declare_model(std::string name, std::string desc)
{
  _add_model(name, desc, [](unsigned LX, unsigned LY, unsigned BC)
             { return ModelPtr(new T(LX, LY, BC)); });
}

ModelPtr NewModel(std::string name, unsigned LX, unsigned LY, unsigned BC);
void ListModels();
void DeclareModels();

#endif
