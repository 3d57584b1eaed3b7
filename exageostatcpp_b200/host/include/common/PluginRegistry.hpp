// Name -> factory registry of kernel plugins
// (inst/include/common/PluginRegistry.hpp:34-94): Add(name, factory) at static
// initialisation, Create(name, timeslot) returns a raw owning pointer.
#pragma once
#include <functional>
#include <map>
#include <stdexcept>
#include <string>

namespace exageostat::plugins {

template <typename T>
class PluginRegistry {
 public:
  using FactoryFunction = std::function<T*()>;
  using FactoryMap = std::map<std::string, FactoryFunction>;

  static bool Add(const std::string& aName, FactoryFunction aFactory) {
    auto& map = GetFactoryMap();
    if (map.find(aName) != map.end()) return false;
    map[aName] = std::move(aFactory);
    return true;
  }

  static T* Create(const std::string& aName, const int& aTimeSlot = 1) {
    (void)aTimeSlot;
    auto& map = GetFactoryMap();
    auto it = map.find(aName);
    if (it == map.end()) throw std::runtime_error("Couldn't create kernel: " + aName + " is not registered");
    return it->second();
  }

  static FactoryMap& GetFactoryMap() {
    static FactoryMap map;
    return map;
  }
};

}  // namespace exageostat::plugins
