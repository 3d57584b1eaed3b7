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

  // ChameleonImplementation<T>::ExaGeoStatLapackCopyTile (ChameleonImplementation.cpp:329-335):
  // the copies the evaluation makes, Z -> Zcpy (first evaluation, :113-119) and
  // Zcpy -> Z (later ones, :120-124), on the data set's device problem.
  void ExaGeoStatLapackCopyTile(const common::UpperLower& aUpperLower, void* apA, void* apB) override {
    (void)aUpperLower;  // vectors: every part is copied
    auto* a = this->View(apA, common::DESCRIPTOR_Z, "ExaGeoStatLapackCopyTile", true);
    auto* b = this->View(apB, common::DESCRIPTOR_Z, "ExaGeoStatLapackCopyTile", true);
    this->SameProblem(a, b, "ExaGeoStatLapackCopyTile");
    if (a->name == common::DESCRIPTOR_Z && b->name == common::DESCRIPTOR_Z_COPY)
      dataunits::EgsCheck(egs_save_observations(a->problem), "egs_save_observations");
    else if (a->name == common::DESCRIPTOR_Z_COPY && b->name == common::DESCRIPTOR_Z)
      dataunits::EgsCheck(egs_restore_observations(a->problem), "egs_restore_observations");
    else
      throw std::domain_error("ExaGeoStatLapackCopyTile: the device copies Z <-> Zcpy");
  }

  // ChameleonImplementation<T>::ExaGeoStatSequenceWait / ExaGeoStatCreateSequence
  // (CHAMELEON_Sequence_Wait / _Create): a sequence is a CUDA stream of the library.
  void ExaGeoStatSequenceWait(void* apSequence) override {
    dataunits::EgsCheck(egs_sequence_wait(apSequence), "egs_sequence_wait");
  }
  void ExaGeoStatCreateSequence(void* apSequence) override {
    dataunits::EgsCheck(egs_sequence_create(static_cast<void**>(apSequence)), "egs_sequence_create");
  }

  // ChameleonDense<T>::ExaGeoStatPotrfTile (ChameleonDense.cpp:25-37): lower Cholesky of
  // the covariance in place; like the dense reference it ignores the band and the
  // low-rank arguments (the data set's band approximation, when set, applies).
  // A non-SPD matrix throws "Matrix is not positive definite" (:29-32).
  void ExaGeoStatPotrfTile(const common::UpperLower& aUpperLower, void* apA, int aBand, void* apCD, void* apCrk,
                           const int& aMaxRank, const int& aAcc) override {
    (void)aBand, (void)apCD, (void)apCrk, (void)aMaxRank, (void)aAcc;
    if (aUpperLower != common::EXAGEOSTAT_LOWER)
      throw std::domain_error("the device factorisation is lower (EXAGEOSTAT_LOWER)");
    auto* a = this->View(apA, common::DESCRIPTOR_C, "ExaGeoStatPotrfTile");
    dataunits::EgsCheck(egs_potrf(a->problem), "egs_potrf");
  }

  // ChameleonImplementation<T>::ExaGeoStatTrsmTile (ChameleonImplementation.cpp:337-347):
  // Z := op(L)^-1 Z with the factor of the same data set; the forms the reference
  // uses (left, lower, non-unit, alpha 1), op = identity or transpose.
  void ExaGeoStatTrsmTile(const common::Side& aSide, const common::UpperLower& aUpperLower,
                          const common::Trans& aTrans, const common::Diag& aDiag, const T& aAlpha, void* apA,
                          void* apCD, void* apCrk, void* apZ, const int& aMaxRank) override {
    (void)apCD, (void)apCrk, (void)aMaxRank;
    if (aSide != common::EXAGEOSTAT_LEFT || aUpperLower != common::EXAGEOSTAT_LOWER ||
        aDiag != common::EXAGEOSTAT_NON_UNIT || aAlpha != T(1) || aTrans == common::EXAGEOSTAT_CONJ_TRANS)
      throw std::domain_error("the device solve is left, lower, non-unit, alpha 1, with or without transpose");
    auto* a = this->View(apA, common::DESCRIPTOR_C, "ExaGeoStatTrsmTile");
    auto* z = this->View(apZ, common::DESCRIPTOR_Z, "ExaGeoStatTrsmTile");
    this->SameProblem(a, z, "ExaGeoStatTrsmTile");
    if (aTrans == common::EXAGEOSTAT_NO_TRANS)
      dataunits::EgsCheck(egs_trsv(a->problem), "egs_trsv");
    else
      dataunits::EgsCheck(egs_trsv_transpose(a->problem), "egs_trsv_transpose");
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
