// Synthetic data generator (src/data-generators/concrete/runtime/StarpuGenerator.cpp:33-89):
// jittered-grid locations from the C library's rand() (LocationGenerator.cpp:25-123)
// and Z = L e on the device.
#pragma once
#include <memory>
#include "configurations/Configurations.hpp"
#include "data-units/ExaGeoStatData.hpp"
#include "linear-algebra-solvers/LinearAlgebraFactory.hpp"

namespace exageostat::generators {

template <typename T>
class SyntheticGenerator {
 public:
  // Locations only; like the reference, continues the global rand() sequence (the API seeds it).
  static void GenerateLocations(const int& aN, dataunits::Locations<T>& aLocations) {
    aLocations.SetSize(aN);
    dataunits::EgsCheck(egs_generate_locations(aN, 0, 0, aLocations.GetLocationX(), aLocations.GetLocationY()),
                        "egs_generate_locations");
  }

  static std::unique_ptr<dataunits::ExaGeoStatData<T>> CreateData(configurations::Configurations& aConfigurations,
                                                                  const kernels::Kernel<T>& aKernel) {
    const int n = aConfigurations.GetProblemSize();
    auto data = std::make_unique<dataunits::ExaGeoStatData<T>>(n, aConfigurations.GetDimension());
    GenerateLocations(n, *data->GetLocations());
    auto solver = linearAlgebra::LinearAlgebraFactory<T>::CreateLinearAlgebraSolver(aConfigurations.GetComputation());
    solver->GenerateSyntheticData(aConfigurations, data, aKernel);
    return data;
  }
};

}  // namespace exageostat::generators
