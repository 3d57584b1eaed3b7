// EXACT_DENSE backend on the B200 library: the drop-in for ChameleonDense<T> /
// ChameleonImplementation<T> (src/linear-algebra-solvers/concrete/chameleon/).
// Device state lives in the data's DescriptorData, because the reference creates
// a new solver object for every NLopt evaluation (StarpuRuntimeSolver.cpp:77-78).
#pragma once
#include <cstdio>
#include <iomanip>
#include <iostream>
#include <vector>
#include "linear-algebra-solvers/LinearAlgebraMethods.hpp"
#include "results/Results.hpp"

namespace exageostat::linearAlgebra {

template <typename T>
class CudaDense : public LinearAlgebraMethods<T> {
 public:
  // ChameleonImplementation<T>::ExaGeoStatMLETile (ChameleonImplementation.cpp:35-327).
  T ExaGeoStatMLETile(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                      configurations::Configurations& aConfigurations, const double* theta, T* apMeasurementsMatrix,
                      const kernels::Kernel<T>& aKernel) override {
    static_assert(sizeof(T) == sizeof(double), "the device path is FP64");
    const int n = aConfigurations.GetProblemSize();
    auto* dd = aData->GetDescriptorData();
    // --precision: MIXED keeps the diagonal and MixedPrecisionBand tile rows in FP64
    // and the other tiles in FP32 (Definitions.hpp Precision; the reference declares
    // the option without a dense mixed implementation)
    const bool mixed = aConfigurations.GetPrecision() == common::MIXED;
    if (mixed && aConfigurations.GetComputation() == common::DIAGONAL_APPROX)
      throw std::domain_error("--precision=mixed and --computation=diag_approx are exclusive");
    const int precision = mixed ? EGS_PRECISION_MIXED : EGS_PRECISION_DOUBLE;
    const int mband = mixed ? aConfigurations.GetMixedPrecisionBand() : 0;
    bool created = false;
    egs_problem* p = dd->EnsureProblem(n, aConfigurations.GetDenseTileSize(), precision, mband, &created);
    if (!mixed) {
      // DIAGONAL_APPROX: ChameleonDST with --band (a band of 0 or 1 keeps only the diagonal tiles)
      const int band = aConfigurations.GetComputation() == common::DIAGONAL_APPROX
                           ? (aConfigurations.GetBand() > 1 ? aConfigurations.GetBand() : 1)
                           : 0;
      dataunits::EgsCheck(egs_problem_set_band(p, band), "egs_problem_set_band");
    }
    if (aData->GetMleIterations() == 0 || created) {
      // first evaluation: upload locations and save Z into Zcpy (:113-119)
      dataunits::EgsCheck(egs_problem_set_locations(p, aData->GetLocations()->GetLocationX(),
                                                    aData->GetLocations()->GetLocationY()),
                          "egs_problem_set_locations");
      std::vector<T>& zc = dd->HostVector(common::DESCRIPTOR_Z_COPY);
      if (apMeasurementsMatrix) {
        zc.assign(apMeasurementsMatrix, apMeasurementsMatrix + n);
      } else {
        zc = dd->HostVector(common::DESCRIPTOR_Z);
        if ((int)zc.size() < n) throw std::runtime_error("no observations for the modeling step");
      }
      dataunits::EgsCheck(egs_problem_set_observations(p, zc.data()), "egs_problem_set_observations");
    }
    double loglik = 0, logdet = 0, dot = 0;
    dataunits::EgsCheck(egs_mle_eval(p, theta, &loglik, &logdet, &dot), "egs_mle_eval");
    const int iter = aData->GetMleIterations();
    if (configurations::Configurations::GetVerbosity() != common::QUIET_MODE) {
      std::cout << "\t" << iter + 1 << " - Model Parameters (";
      for (int i = 0; i < aKernel.GetParametersNumbers(); ++i)
        std::cout << std::setprecision(8) << theta[i] << (i + 1 < aKernel.GetParametersNumbers() ? ", " : "");
      std::cout << ")----> LogLi: " << std::setprecision(18) << loglik << "\n";
    }
    aData->SetMleIterations(iter + 1);
    auto* res = results::Results::GetInstance();
    res->SetMLEIterations(iter + 1);
    res->SetMaximumTheta(std::vector<double>(theta, theta + aKernel.GetParametersNumbers()));
    res->SetLogLikValue(loglik);
    return loglik;
  }

  // LinearAlgebraMethods<T>::GenerateSyntheticData / GenerateObservationsVector
  // (LinearAlgebraMethods.cpp:322-449): Z = L e at the initial theta, e = DLARNV(3, {s,s,s,1}).
  void GenerateSyntheticData(configurations::Configurations& aConfigurations,
                             std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                             const kernels::Kernel<T>& aKernel) override {
    (void)aKernel;
    const int n = aConfigurations.GetProblemSize();
    auto* dd = aData->GetDescriptorData();
    egs_problem* p = dd->EnsureProblem(n, aConfigurations.GetDenseTileSize());
    dataunits::EgsCheck(egs_problem_set_locations(p, aData->GetLocations()->GetLocationX(),
                                                  aData->GetLocations()->GetLocationY()),
                        "egs_problem_set_locations");
    std::vector<T>& z = dd->HostVector(common::DESCRIPTOR_Z);
    z.assign(n, 0.0);
    dataunits::EgsCheck(egs_generate_observations(p, aConfigurations.GetInitialTheta().data(),
                                                  aConfigurations.GetSeed(), z.data()),
                        "egs_generate_observations");
    results::Results::GetInstance()->SetGeneratedLocationsNumber(n);
  }

  // LinearAlgebraMethods<T>::ExaGeoStatMLEPredictTile (LinearAlgebraMethods.cpp:451-605).
  T* ExaGeoStatMLEPredictTile(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData, T* apTheta,
                              const int& aZMissNumber, const int& aZObsNumber, T* apZObs, T* apZActual, T* apZMiss,
                              configurations::Configurations& aConfiguration, dataunits::Locations<T>& aMissLocations,
                              dataunits::Locations<T>& aObsLocations, const kernels::Kernel<T>& aKernel) override {
    (void)aData;
    (void)aKernel;
    double mspe = -1;
    dataunits::EgsCheck(
        egs_predict_host(aZObsNumber, aZMissNumber, aConfiguration.GetDenseTileSize(), aObsLocations.GetLocationX(),
                         aObsLocations.GetLocationY(), apZObs, aMissLocations.GetLocationX(),
                         aMissLocations.GetLocationY(), apZActual, apTheta, apZMiss, &mspe),
        "egs_predict_host");
    results::Results::GetInstance()->SetMSPEError(mspe);
    T* all = new T[3];
    all[0] = mspe;
    all[1] = apZActual ? 0 : -1;
    all[2] = apZActual ? 0 : -1;
    return all;
  }
};

}  // namespace exageostat::linearAlgebra
