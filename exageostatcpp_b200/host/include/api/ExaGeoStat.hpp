// Public facade (inst/include/api/ExaGeoStat.hpp:28-86, src/api/ExaGeoStat.cpp:72-125):
// generate/load data, model (MLE fit), predict.
#pragma once
#include "data-loader/CSVLoader.hpp"
#include <cstdlib>
#include <memory>
#include "configurations/Configurations.hpp"
#include "data-generators/SyntheticGenerator.hpp"
#include "data-units/ExaGeoStatData.hpp"
#include "kernels/concrete/UnivariateMaternStationary.hpp"
#include "prediction/Prediction.hpp"
#include "runtime-solver/RuntimeSolver.hpp"

namespace exageostat::api {

template <typename T>
class ExaGeoStat {
 public:
  // ExaGeoStat.cpp:72-88: srand(seed), then locations and Z = L e at the initial theta.
  static void ExaGeoStatLoadData(configurations::Configurations& aConfigurations,
                                 std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData) {
    // --datapath: the CSV loader (DataLoader.cpp:29, CSVLoader.cpp:37-143); else synthetic data
    if (!aConfigurations.GetDataPath().empty()) {
      aData = dataLoader::csv::CSVLoader<T>::LoadData(aConfigurations);
      return;
    }
    std::srand(aConfigurations.GetSeed());
    std::unique_ptr<kernels::Kernel<T>> kernel(plugins::PluginRegistry<kernels::Kernel<T>>::Create(
        aConfigurations.GetKernelName(), aConfigurations.GetTimeSlot()));
    aData = generators::SyntheticGenerator<T>::CreateData(aConfigurations, *kernel);
  }

  // ExaGeoStat.cpp:90-107.
  static T ExaGeoStatDataModeling(configurations::Configurations& aConfigurations,
                                  std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                                  T* apMeasurementsMatrix = nullptr) {
    std::unique_ptr<kernels::Kernel<T>> kernel(plugins::PluginRegistry<kernels::Kernel<T>>::Create(
        aConfigurations.GetKernelName(), aConfigurations.GetTimeSlot()));
    aConfigurations.InitializeAllTheta();
    runtimesolver::RuntimeSolver<T> solver;
    return solver.ModelingOperations(aData, aConfigurations, apMeasurementsMatrix, *kernel);
  }

  // ExaGeoStat.cpp:110-125.
  static void ExaGeoStatPrediction(configurations::Configurations& aConfigurations,
                                   std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                                   T* apMeasurementsMatrix = nullptr,
                                   dataunits::Locations<T>* apTrainLocations = nullptr,
                                   dataunits::Locations<T>* apTestLocations = nullptr) {
    std::unique_ptr<kernels::Kernel<T>> kernel(plugins::PluginRegistry<kernels::Kernel<T>>::Create(
        aConfigurations.GetKernelName(), aConfigurations.GetTimeSlot()));
    aConfigurations.InitializeAllTheta();
    prediction::Prediction<T>::PredictMissingData(aData, aConfigurations, apMeasurementsMatrix, *kernel,
                                                  apTrainLocations, apTestLocations);
  }
};

}  // namespace exageostat::api
