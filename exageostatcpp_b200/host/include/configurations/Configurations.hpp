// Run configuration of the MLE path (src/configurations/Configurations.cpp).
// Setters/getters keep the reference's names and meaning: SetTolerance(k)
// stores 10^-k (:380-382), InitializeAllTheta starts the optimiser at the lower
// bounds and pins parameters whose estimated value is not -1 (:182-213),
// CalculateZObsNumber = N - ZMiss (:364-366).  Defaults follow
// configurations/config.json (N 16, dts 8, max MLE iterations 1, tolerance 1,
// seed 0).
#pragma once
#include <cmath>
#include <string>
#include <vector>
#include "common/Definitions.hpp"

namespace exageostat::configurations {

class Configurations {
 public:
  Configurations() = default;

  // Command-line form "--key=value" (keys normalised like Parser::ProcessKeyString,
  // src/configurations/Parser.cpp:70-81: lower case, alphanumerics only); theta
  // lists use ':' and "?" for a free parameter (-1), Validator.cpp:209-255.
  void InitializeArguments(const int& argc, char** argv);

#define EGS_PROP(Type, Name, Init)                       \
 public:                                                 \
  void Set##Name(const Type& aValue) { m##Name = aValue; } \
  Type Get##Name() const { return m##Name; }             \
                                                         \
 private:                                                \
  Type m##Name = Init;

  EGS_PROP(int, ProblemSize, 16)
  EGS_PROP(std::string, KernelName, "UnivariateMaternStationary")
  EGS_PROP(int, DenseTileSize, 8)
  EGS_PROP(int, LowTileSize, 0)
  EGS_PROP(common::Computation, Computation, common::EXACT_DENSE)
  EGS_PROP(common::Dimension, Dimension, common::Dimension2D)
  EGS_PROP(common::Precision, Precision, common::DOUBLE)
  EGS_PROP(int, Seed, 0)
  EGS_PROP(int, MaxMleIterations, 1)
  EGS_PROP(int, UnknownObservationsNb, 0)
  EGS_PROP(int, ObservationNumber, 0)
  EGS_PROP(int, TimeSlot, 1)
  EGS_PROP(int, Band, 0)
  EGS_PROP(int, MixedPrecisionBand, 2)  // FP64 tile rows below the diagonal with --precision=mixed
  EGS_PROP(int, MaxRank, 0)
  EGS_PROP(int, CoresNumber, 1)
  EGS_PROP(int, GPUsNumbers, 1)
  EGS_PROP(int, DistanceMetric, common::EUCLIDEAN_DISTANCE)
  EGS_PROP(bool, IsMSPE, false)
  EGS_PROP(bool, IsIDW, false)
  EGS_PROP(bool, IsFisher, false)
  EGS_PROP(bool, IsMLOEMMOM, false)
  EGS_PROP(bool, IsNonGaussian, false)
  EGS_PROP(std::string, RecoveryFile, "")
  EGS_PROP(std::string, DataPath, "")  // CSV data file (--datapath); empty: synthetic data
#undef EGS_PROP

 public:
  void SetTolerance(double aExponent) { mTolerance = std::pow(10.0, -1.0 * aExponent); }
  double GetTolerance() const { return mTolerance; }

  void SetInitialTheta(const std::vector<double>& v) { mInitialTheta = v; }
  std::vector<double>& GetInitialTheta() { return mInitialTheta; }
  void SetLowerBounds(const std::vector<double>& v) { mLowerBounds = v; }
  std::vector<double>& GetLowerBounds() { return mLowerBounds; }
  void SetUpperBounds(const std::vector<double>& v) { mUpperBounds = v; }
  std::vector<double>& GetUpperBounds() { return mUpperBounds; }
  void SetStartingTheta(const std::vector<double>& v) { mStartingTheta = v; }
  std::vector<double>& GetStartingTheta() { return mStartingTheta; }
  void SetEstimatedTheta(const std::vector<double>& v) { mEstimatedTheta = v; }
  std::vector<double>& GetEstimatedTheta() { return mEstimatedTheta; }

  int CalculateZObsNumber() { return GetProblemSize() - GetUnknownObservationsNb(); }
  void InitializeAllTheta();
  void PrintSummary() {}

  static void SetVerbosity(const common::Verbose& aVerbose) { Verbosity() = aVerbose; }
  static common::Verbose GetVerbosity() { return Verbosity(); }

 private:
  static common::Verbose& Verbosity() {
    static common::Verbose v = common::STANDARD_MODE;
    return v;
  }
  static void InitTheta(std::vector<double>& aTheta, int size);

  double mTolerance = 0.1;
  std::vector<double> mInitialTheta, mLowerBounds, mUpperBounds, mStartingTheta, mEstimatedTheta;
  bool mIsThetaInit = false;
};

}  // namespace exageostat::configurations
