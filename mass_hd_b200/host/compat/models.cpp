// Name registry of the standalone plugin build (reference: src/models.cpp).
#include "models.hpp"
#include "error_msg.hpp"

#include <map>

namespace {
struct FactoryAndDesc
{
  std::string desc;
  Factory fact;
};
std::map<std::string, FactoryAndDesc>& registry()
{
  static std::map<std::string, FactoryAndDesc> m;
  return m;
}
}

void _add_model(std::string name, std::string desc, Factory fact)
{
  if(registry().count(name)) throw error_msg("model '", name, "' already registered.");
  registry()[name] = {desc, fact};
}

ModelPtr NewModel(std::string name, unsigned LX, unsigned LY, unsigned BC)
{
  auto it = registry().find(name);
  if(it == registry().end())
    throw error_msg("model '", name, "' can not be found. Type --list for a list of available models.");
  return it->second.fact(LX, LY, BC);
}

void ListModels()
{
  for(const auto& m : registry())
    std::cout << '\n' << m.first << ":\n" << std::string(m.first.size() + 1, '-') << '\n'
              << m.second.desc << '\n';
}
