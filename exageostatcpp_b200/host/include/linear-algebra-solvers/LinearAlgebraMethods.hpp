// The linear-algebra seam of the MLE path
// (inst/include/linear-algebra-solvers/LinearAlgebraMethods.hpp:50-401).  Kept
// members: ExaGeoStatMLETile (one log-likelihood evaluation), the synthetic-data
// generator, kriging (ExaGeoStatMLEPredictTile) and ExaGeoStatGetZObs.  The only
// concrete backend is CudaDense<T> (the B200 library, EXACT_DENSE).
#pragma once
#include <memory>
#include <vector>
#include "configurations/Configurations.hpp"
#include "data-units/ExaGeoStatData.hpp"
#include "kernels/Kernel.hpp"

namespace exageostat::linearAlgebra {

template <typename T>
class LinearAlgebraMethods {
 public:
  virtual ~LinearAlgebraMethods() = default;

  virtual T ExaGeoStatMLETile(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                              configurations::Configurations& aConfigurations, const double* theta,
                              T* apMeasurementsMatrix, const kernels::Kernel<T>& aKernel) = 0;

  virtual void GenerateSyntheticData(configurations::Configurations& aConfigurations,
                                     std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                                     const kernels::Kernel<T>& aKernel) = 0;

  // Returns new T[3] = {mspe, mspe1, mspe2} (LinearAlgebraMethods.cpp:597-603);
  // mspe is -1 when apZActual is null (:579-581).
  virtual T* ExaGeoStatMLEPredictTile(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData, T* apTheta,
                                      const int& aZMissNumber, const int& aZObsNumber, T* apZObs, T* apZActual,
                                      T* apZMiss, configurations::Configurations& aConfiguration,
                                      dataunits::Locations<T>& aMissLocations, dataunits::Locations<T>& aObsLocations,
                                      const kernels::Kernel<T>& aKernel) = 0;

  // Copy of the observations: the caller's measurements when given, else the data's Z
  // (LinearAlgebraMethods.cpp:1308-1340).
  void ExaGeoStatGetZObs(configurations::Configurations& aConfigurations, T* apZ, const int& aSize,
                         dataunits::DescriptorData<T>& aDescData, T* apMeasurementsMatrix, const int& aP) {
    (void)aConfigurations;
    (void)aP;
    if (apMeasurementsMatrix) {
      for (int i = 0; i < aSize; ++i) apZ[i] = apMeasurementsMatrix[i];
      return;
    }
    auto& z = aDescData.HostVector(common::DESCRIPTOR_Z);
    if ((int)z.size() < aSize) throw std::runtime_error("no observations: pass a measurements vector or generate data");
    for (int i = 0; i < aSize; ++i) apZ[i] = z[i];
  }
};

}  // namespace exageostat::linearAlgebra
