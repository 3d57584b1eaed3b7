// Kriging dispatcher (src/prediction/Prediction.cpp:33-241) and its random
// hold-out split (src/prediction/PredictionHelpers.cpp:23-168).  Without explicit
// train/test locations, ZMiss points are held out by a Fisher-Yates shuffle that
// draws from the C library's rand() (j = i + rand() / (RAND_MAX/(n-i) + 1), :146);
// with explicit locations the MSPE is reported as -1 (no truth).
#pragma once
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <vector>
#include "configurations/Configurations.hpp"
#include "data-units/ExaGeoStatData.hpp"
#include "linear-algebra-solvers/LinearAlgebraFactory.hpp"
#include "results/Results.hpp"

namespace exageostat::prediction {

template <typename T>
class PredictionHelpers {
 public:
  // PredictionHelpers<T>::Shuffle (PredictionHelpers.cpp:140-168), univariate 2-D case.
  static void Shuffle(T* apArray, dataunits::Locations<T>& aLocations, int aSize) {
    if (aSize > 1) {
      for (size_t i = 0; i < (size_t)aSize - 1; i++) {
        size_t j = i + rand() / (RAND_MAX / (aSize - i) + 1);
        std::swap(apArray[j], apArray[i]);
        std::swap(aLocations.GetLocationX()[j], aLocations.GetLocationX()[i]);
        std::swap(aLocations.GetLocationY()[j], aLocations.GetLocationY()[i]);
      }
    }
  }

  // PickRandomPoints (PredictionHelpers.cpp:23-138) for p = 1: shuffle Z with the
  // locations, the first ZMiss entries are the held-out truth, the rest observed.
  static void PickRandomPoints(configurations::Configurations& aConfigurations,
                               std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData, T* apZObs, T* apZActual, T* apZ,
                               dataunits::Locations<T>& aMissLocation, dataunits::Locations<T>& aObsLocation) {
    const int n = aConfigurations.GetProblemSize();
    const int nmiss = aConfigurations.GetUnknownObservationsNb();
    const int nobs = aConfigurations.CalculateZObsNumber();
    dataunits::Locations<T> l(n, aData->GetLocations()->GetDimension());
    for (int i = 0; i < n; ++i) {
      l.GetLocationX()[i] = aData->GetLocations()->GetLocationX()[i];
      l.GetLocationY()[i] = aData->GetLocations()->GetLocationY()[i];
    }
    Shuffle(apZ, l, n);
    for (int i = 0; i < nmiss; ++i) {
      apZActual[i] = apZ[i];
      aMissLocation.GetLocationX()[i] = l.GetLocationX()[i];
      aMissLocation.GetLocationY()[i] = l.GetLocationY()[i];
    }
    for (int i = 0; i < nobs; ++i) {
      apZObs[i] = apZ[nmiss + i];
      aObsLocation.GetLocationX()[i] = l.GetLocationX()[nmiss + i];
      aObsLocation.GetLocationY()[i] = l.GetLocationY()[nmiss + i];
    }
  }
};

template <typename T>
class Prediction {
 public:
  static void PredictMissingData(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                                 configurations::Configurations& aConfigurations, T* apMeasurementsMatrix,
                                 const kernels::Kernel<T>& aKernel, dataunits::Locations<T>* apTrainLocations = nullptr,
                                 dataunits::Locations<T>* apTestLocations = nullptr) {
    const int np = aKernel.GetParametersNumbers();
    std::vector<double>& et = aConfigurations.GetEstimatedTheta();
    bool can_predict = (int)et.size() >= np;
    for (int i = 0; can_predict && i < np; ++i)
      if (et[i] == -1) can_predict = false;
    if (!can_predict && (aConfigurations.GetIsMLOEMMOM() || aConfigurations.GetIsMSPE() || aConfigurations.GetIsFisher()))
      throw std::runtime_error(
          "Can't predict without an estimated theta, please either pass --etheta or run the modeling module before "
          "prediction");
    int nmiss, nobs;
    bool truth;
    if (!apTrainLocations && !apTestLocations) {
      nmiss = aConfigurations.GetUnknownObservationsNb();
      nobs = aConfigurations.CalculateZObsNumber();
      truth = true;
    } else {
      nmiss = apTestLocations->GetSize();
      nobs = apTrainLocations->GetSize();
      truth = false;
    }
    aConfigurations.SetObservationNumber(nobs);
    // Fisher information on all locations (Prediction.cpp:76-87), before the split
    if (aConfigurations.GetIsFisher()) {
      std::vector<double> fisher(9);
      dataunits::EgsCheck(egs_fisher_host(aConfigurations.GetProblemSize(), aConfigurations.GetDenseTileSize(),
                                          aData->GetLocations()->GetLocationX(), aData->GetLocations()->GetLocationY(),
                                          et.data(), fisher.data()),
                          "egs_fisher_host");
      results::Results::GetInstance()->SetFisherMatrix(fisher);
    }
    if (nmiss <= 0) return;
    results::Results::GetInstance()->SetZMiss(nmiss);
    auto solver = linearAlgebra::LinearAlgebraFactory<T>::CreateLinearAlgebraSolver(common::EXACT_DENSE);
    std::vector<T> zobs(nobs), zmiss(nmiss), zactual(truth ? nmiss : 0);
    dataunits::Locations<T> miss(nmiss, aConfigurations.GetDimension()), obs(nobs, aConfigurations.GetDimension());
    // InitializePredictionArguments (Prediction.cpp:213-241)
    const int n = aConfigurations.GetProblemSize();
    std::vector<T> z(truth ? n : nobs);
    if (truth) {
      solver->ExaGeoStatGetZObs(aConfigurations, z.data(), n, *aData->GetDescriptorData(), apMeasurementsMatrix, 1);
      PredictionHelpers<T>::PickRandomPoints(aConfigurations, aData, zobs.data(), zactual.data(), z.data(), miss, obs);
    } else {
      for (int i = 0; i < nobs; ++i) {
        obs.GetLocationX()[i] = apTrainLocations->GetLocationX()[i];
        obs.GetLocationY()[i] = apTrainLocations->GetLocationY()[i];
      }
      for (int i = 0; i < nmiss; ++i) {
        miss.GetLocationX()[i] = apTestLocations->GetLocationX()[i];
        miss.GetLocationY()[i] = apTestLocations->GetLocationY()[i];
      }
      solver->ExaGeoStatGetZObs(aConfigurations, zobs.data(), nobs, *aData->GetDescriptorData(), apMeasurementsMatrix,
                                1);
    }
    // MLOE / MMOM with the initial theta as the truth (Prediction.cpp:132-139)
    if (aConfigurations.GetIsMLOEMMOM()) {
      double mloe = 0, mmom = 0;
      dataunits::EgsCheck(egs_mloe_mmom_host(nobs, nmiss, aConfigurations.GetDenseTileSize(), obs.GetLocationX(),
                                             obs.GetLocationY(), miss.GetLocationX(), miss.GetLocationY(),
                                             aConfigurations.GetInitialTheta().data(), et.data(), &mloe, &mmom),
                          "egs_mloe_mmom_host");
      results::Results::GetInstance()->SetMLOE(mloe);
      results::Results::GetInstance()->SetMMOM(mmom);
    }
    if (aConfigurations.GetIsMSPE()) {
      T* err = solver->ExaGeoStatMLEPredictTile(aData, et.data(), nmiss, nobs, zobs.data(),
                                                truth ? zactual.data() : nullptr, zmiss.data(), aConfigurations, miss,
                                                obs, aKernel);
      delete[] err;
      results::Results::GetInstance()->SetPredictedMissedValues(std::vector<double>(zmiss.begin(), zmiss.end()));
    }
  }
};

}  // namespace exageostat::prediction
