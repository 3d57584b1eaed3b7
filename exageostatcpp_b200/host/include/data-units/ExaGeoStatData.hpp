// Owner of the locations and descriptors of one data set
// (src/data-units/ExaGeoStatData.cpp:21-113), plus the MLE iteration counter that
// ExaGeoStatMLETile uses to decide between saving and restoring Z.
#pragma once
#include <memory>
#include "data-units/DescriptorData.hpp"
#include "data-units/Locations.hpp"

namespace exageostat::dataunits {

template <typename T>
class ExaGeoStatData {
 public:
  ExaGeoStatData(const int& aSize, const common::Dimension& aDimension)
      : mLocations(new Locations<T>(aSize, aDimension)), mDescriptorData(new DescriptorData<T>()) {}

  Locations<T>* GetLocations() { return mLocations.get(); }
  // Takes ownership, like ExaGeoStatData::SetLocations (ExaGeoStatData.cpp:45-57).
  void SetLocations(Locations<T>& aLocation) { mLocations.reset(&aLocation); }
  DescriptorData<T>* GetDescriptorData() { return mDescriptorData.get(); }
  int GetMleIterations() const { return mMleIterations; }
  void SetMleIterations(const int& aIterations) { mMleIterations = aIterations; }

 private:
  std::unique_ptr<Locations<T>> mLocations;
  std::unique_ptr<DescriptorData<T>> mDescriptorData;
  int mMleIterations = 0;
};

}  // namespace exageostat::dataunits
