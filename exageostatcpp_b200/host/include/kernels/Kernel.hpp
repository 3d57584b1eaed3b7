// Covariance-kernel plugin interface (inst/include/kernels/Kernel.hpp:69-128):
// GenerateCovarianceMatrix fills a rows x cols column-major block
// A[i + j*rows] for locations i0 = row offset .., j0 = column offset ...
#pragma once
#include <string>
#include <unordered_map>
#include "common/PluginRegistry.hpp"
#include "data-units/Locations.hpp"

namespace exageostat::kernels {

struct KernelsConfigurations {
  static std::unordered_map<std::string, int>& GetParametersNumberKernelMap() {
    static std::unordered_map<std::string, int> map;
    return map;
  }
};

template <typename T>
class Kernel {
 public:
  virtual ~Kernel() = default;
  virtual void GenerateCovarianceMatrix(T* apMatrixA, const int& aRowsNumber, const int& aColumnsNumber,
                                        const int& aRowOffset, const int& aColumnOffset,
                                        dataunits::Locations<T>& aLocation1, dataunits::Locations<T>& aLocation2,
                                        dataunits::Locations<T>& aLocation3, T* aLocalTheta,
                                        const int& aDistanceMetric) = 0;
  virtual std::string GetKernelName() const = 0;
  int GetVariablesNumber() const { return mP; }
  int GetParametersNumbers() const { return mParametersNumber; }

 protected:
  int mP = 1;
  int mParametersNumber = 0;
};

}  // namespace exageostat::kernels
