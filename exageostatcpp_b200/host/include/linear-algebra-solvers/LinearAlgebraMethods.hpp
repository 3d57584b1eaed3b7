// The linear-algebra seam of the MLE path
// (inst/include/linear-algebra-solvers/LinearAlgebraMethods.hpp:50-401).  Kept
// members: the descriptor set-up (InitiateDescriptors), ExaGeoStatMLETile (one
// log-likelihood evaluation), the synthetic-data generator, the tile operations
// the reference declares pure virtual (LapackCopyTile, SequenceWait,
// CreateSequence, PotrfTile, TrsmTile), the dposv solve, the copies between
// LAPACK and descriptor layouts, kriging (ExaGeoStatMLEPredictTile) and
// ExaGeoStatGetZObs.  The only concrete backend is CudaDense<T> (the B200
// library, EXACT_DENSE).
//
// A descriptor handle (void* apA, apZ, ...) is the DescriptorView that
// DescriptorData::GetDescriptor returns (its chameleon_desc / cuda_desc): it names
// one matrix (C, Z, Zcpy) of the device problem that holds the data set.
#pragma once
#include <algorithm>
#include <memory>
#include <stdexcept>
#include <vector>
#include "configurations/Configurations.hpp"
#include "data-units/ExaGeoStatData.hpp"
#include "kernels/Kernel.hpp"

namespace exageostat::linearAlgebra {

template <typename T>
class LinearAlgebraMethods {
 public:
  virtual ~LinearAlgebraMethods() = default;

  // LinearAlgebraMethods<T>::InitiateDescriptors (LinearAlgebraMethods.hpp:62-64,
  // LinearAlgebraMethods.cpp:36-118): the descriptors of one data set -- here the
  // device problem of n points with tile dts in the configured precision -- and Z
  // from the measurements when they are given.
  void InitiateDescriptors(configurations::Configurations& aConfigurations,
                           dataunits::DescriptorData<T>& aDescriptorData, const int& aP,
                           T* apMeasurementsMatrix = nullptr) {
    static_assert(sizeof(T) == sizeof(double), "the device path is FP64");
    if (aP != 1) throw std::domain_error("only univariate kernels (P = 1) are on the device path");
    const bool mixed = aConfigurations.GetPrecision() == common::MIXED;
    egs_problem* p = aDescriptorData.EnsureProblem(aConfigurations.GetProblemSize(),
                                                   aConfigurations.GetDenseTileSize(),
                                                   mixed ? EGS_PRECISION_MIXED : EGS_PRECISION_DOUBLE,
                                                   mixed ? aConfigurations.GetMixedPrecisionBand() : 0);
    if (apMeasurementsMatrix) {
      const int n = aConfigurations.GetProblemSize();
      aDescriptorData.HostVector(common::DESCRIPTOR_Z).assign(apMeasurementsMatrix, apMeasurementsMatrix + n);
      dataunits::EgsCheck(egs_problem_set_observations(p, apMeasurementsMatrix), "egs_problem_set_observations");
    }
  }

  virtual T ExaGeoStatMLETile(std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                              configurations::Configurations& aConfigurations, const double* theta,
                              T* apMeasurementsMatrix, const kernels::Kernel<T>& aKernel) = 0;

  virtual void GenerateSyntheticData(configurations::Configurations& aConfigurations,
                                     std::unique_ptr<dataunits::ExaGeoStatData<T>>& aData,
                                     const kernels::Kernel<T>& aKernel) = 0;

  // Copies matrix A into matrix B in the tile layout (LinearAlgebraMethods.hpp:153).
  virtual void ExaGeoStatLapackCopyTile(const common::UpperLower& aUpperLower, void* apA, void* apB) = 0;
  // Waits for the completion of a sequence (LinearAlgebraMethods.hpp:161).
  virtual void ExaGeoStatSequenceWait(void* apSequence) = 0;
  // Creates a sequence; apSequence points to the handle to fill (LinearAlgebraMethods.hpp:169).
  virtual void ExaGeoStatCreateSequence(void* apSequence) = 0;
  // Cholesky factorisation of the symmetric positive definite A (LinearAlgebraMethods.hpp:184-186).
  virtual void ExaGeoStatPotrfTile(const common::UpperLower& aUpperLower, void* apA, int aBand, void* apCD,
                                   void* apCrk, const int& aMaxRank, const int& aAcc) = 0;
  // op(A) X = alpha B with the triangular A, B overwritten by X (LinearAlgebraMethods.hpp:203-205).
  virtual void ExaGeoStatTrsmTile(const common::Side& aSide, const common::UpperLower& aUpperLower,
                                  const common::Trans& aTrans, const common::Diag& aDiag, const T& aAlpha, void* apA,
                                  void* apCD, void* apCrk, void* apZ, const int& aMaxRank) = 0;

  // A X = B for the symmetric positive definite A, B overwritten by X (dposv,
  // LinearAlgebraMethods.hpp:216): the Cholesky factorisation of A, then
  // B := L^-1 B and B := L^-T B.  A is the covariance, B the observations of the
  // same data set.
  void ExaGeoStatPosvTile(const common::UpperLower& aUpperLower, void* apA, void* apB) {
    if (aUpperLower != common::EXAGEOSTAT_LOWER)
      throw std::domain_error("the device factorisation is lower (EXAGEOSTAT_LOWER)");
    auto* a = View(apA, common::DESCRIPTOR_C, "ExaGeoStatPosvTile");
    auto* b = View(apB, common::DESCRIPTOR_Z, "ExaGeoStatPosvTile");
    SameProblem(a, b, "ExaGeoStatPosvTile");
    dataunits::EgsCheck(egs_potrf(a->problem), "egs_potrf");
    dataunits::EgsCheck(egs_trsv(a->problem), "egs_trsv");
    dataunits::EgsCheck(egs_trsv_transpose(a->problem), "egs_trsv_transpose");
  }

  // Copies a LAPACK (column-major, leading dimension aLDA) matrix into a descriptor
  // (LinearAlgebraMethods.hpp:275).  C: the stored lower tiles take the part of A
  // named by aUpperLower (upper parts transposed), with the identity in the
  // padding; Z: the observations (Z and its saved copy).
  void ExaGeoStatLap2Desc(T* apA, const int& aLDA, void* apDescA, const common::UpperLower& aUpperLower) {
    auto* d = View(apDescA, common::DESCRIPTOR_C, "ExaGeoStatLap2Desc", true);
    if (d->name == common::DESCRIPTOR_Z) {
      dataunits::EgsCheck(egs_problem_set_observations(d->problem, apA), "egs_problem_set_observations");
      return;
    }
    if (d->name != common::DESCRIPTOR_C) throw std::domain_error("ExaGeoStatLap2Desc: C or Z descriptors only");
    int n = 0, ts = 0, nt = 0;
    long long bytes = 0;
    dataunits::EgsCheck(egs_problem_info(d->problem, &n, &ts, &nt, &bytes), "egs_problem_info");
    if (aLDA < n) throw std::invalid_argument("ExaGeoStatLap2Desc: leading dimension below n");
    const bool upper = aUpperLower == common::EXAGEOSTAT_UPPER;
    std::vector<double> tile((size_t)ts * ts);
    for (int j = 0; j < nt; ++j)
      for (int i = j; i < nt; ++i) {
        for (int c = 0; c < ts; ++c)
          for (int r = 0; r < ts; ++r) {
            const long long gr = (long long)i * ts + r, gc = (long long)j * ts + c;
            double v;
            if (gr >= n || gc >= n) v = (gr == gc) ? 1.0 : 0.0;
            else if (gr < gc) v = 0.0;  // above the diagonal of a diagonal tile: not stored
            else v = upper ? apA[gc + gr * (long long)aLDA] : apA[gr + gc * (long long)aLDA];
            tile[r + (size_t)c * ts] = v;
          }
        dataunits::EgsCheck(egs_set_tile(d->problem, i, j, tile.data()), "egs_set_tile");
      }
  }

  // Copies a descriptor into a LAPACK matrix (LinearAlgebraMethods.hpp:286).  C:
  // the lower tiles fill the part of A named by aUpperLower (both triangles for
  // EXAGEOSTAT_UPPER_LOWER); Z: the current observations.
  void ExaGeoStatDesc2Lap(T* apA, const int& aLDA, void* apDescA, const common::UpperLower& aUpperLower) {
    auto* d = View(apDescA, common::DESCRIPTOR_C, "ExaGeoStatDesc2Lap", true);
    if (d->name == common::DESCRIPTOR_Z) {
      dataunits::EgsCheck(egs_get_observations(d->problem, apA), "egs_get_observations");
      return;
    }
    if (d->name != common::DESCRIPTOR_C) throw std::domain_error("ExaGeoStatDesc2Lap: C or Z descriptors only");
    int n = 0, ts = 0, nt = 0;
    long long bytes = 0;
    dataunits::EgsCheck(egs_problem_info(d->problem, &n, &ts, &nt, &bytes), "egs_problem_info");
    if (aLDA < n) throw std::invalid_argument("ExaGeoStatDesc2Lap: leading dimension below n");
    std::vector<double> tile((size_t)ts * ts);
    for (int j = 0; j < nt; ++j)
      for (int i = j; i < nt; ++i) {
        dataunits::EgsCheck(egs_get_tile(d->problem, i, j, tile.data()), "egs_get_tile");
        for (int c = 0; c < ts; ++c)
          for (int r = 0; r < ts; ++r) {
            const long long gr = (long long)i * ts + r, gc = (long long)j * ts + c;
            if (gr >= n || gc >= n || gr < gc) continue;
            const double v = tile[r + (size_t)c * ts];
            if (aUpperLower != common::EXAGEOSTAT_UPPER) apA[gr + gc * (long long)aLDA] = v;
            if (aUpperLower != common::EXAGEOSTAT_LOWER) apA[gc + gr * (long long)aLDA] = v;
          }
      }
  }

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

 protected:
  // The descriptor behind a void* handle, checked against the name the operation needs
  // (any name when aAnyName).
  static dataunits::DescriptorView<T>* View(void* apDesc, common::DescriptorName aName, const char* aWhere,
                                            bool aAnyName = false) {
    auto* d = static_cast<dataunits::DescriptorView<T>*>(apDesc);
    if (!d || !d->problem)
      throw std::invalid_argument(std::string(aWhere) + ": descriptor without a device problem "
                                                        "(call InitiateDescriptors first)");
    if (!aAnyName && d->name != aName) throw std::domain_error(std::string(aWhere) + ": unexpected descriptor");
    return d;
  }
  static void SameProblem(const dataunits::DescriptorView<T>* a, const dataunits::DescriptorView<T>* b,
                          const char* aWhere) {
    if (a->problem != b->problem)
      throw std::domain_error(std::string(aWhere) + ": both descriptors must belong to one data set");
  }
};

}  // namespace exageostat::linearAlgebra
