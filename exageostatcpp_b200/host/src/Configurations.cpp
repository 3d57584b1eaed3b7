// Non-template parts of Configurations (src/configurations/Configurations.cpp,
// Parser.cpp:23-81, Validator.cpp:209-255 for the theta strings,
// Validator.cpp:108-173 and 285-294 for the computation, precision, kernel
// and distance values).
#include "configurations/Configurations.hpp"

#include <cctype>
#include <sstream>
#include <stdexcept>
#include <string>

#include "kernels/Kernel.hpp"

namespace exageostat::configurations {

void Configurations::InitTheta(std::vector<double>& aTheta, int size) {
  if (aTheta.empty()) {
    for (int i = 0; i < size; i++) aTheta.push_back(-1);
  } else if ((int)aTheta.size() < size) {
    for (int i = (int)aTheta.size(); i < size; i++) aTheta.push_back(0);
  }
}

void Configurations::InitializeAllTheta() {
  if (mIsThetaInit) return;
  int np = kernels::KernelsConfigurations::GetParametersNumberKernelMap()[GetKernelName()];
  if (np <= 0) np = 3;
  InitTheta(mInitialTheta, np);
  InitTheta(mLowerBounds, np);
  InitTheta(mUpperBounds, np);
  mStartingTheta = mLowerBounds;
  InitTheta(mEstimatedTheta, np);
  for (int i = 0; i < np; i++) {
    if (mEstimatedTheta[i] != -1) {
      mLowerBounds[i] = mEstimatedTheta[i];
      mUpperBounds[i] = mEstimatedTheta[i];
      mStartingTheta[i] = mEstimatedTheta[i];
    }
  }
  mIsThetaInit = true;
}

namespace {

std::string normalise_key(const std::string& key) {
  std::string out;
  for (char c : key)
    if (std::isalnum((unsigned char)c)) out += (char)std::tolower((unsigned char)c);
  return out;
}

std::vector<double> parse_theta(const std::string& v) {
  std::vector<double> out;
  std::stringstream ss(v);
  std::string item;
  while (std::getline(ss, item, ':')) out.push_back(item == "?" ? -1.0 : std::stod(item));
  return out;
}

bool parse_bool(const std::string& v) { return v == "true" || v == "1" || v == "TRUE" || v == "True"; }

// Validator::CheckKernelValue (Validator.cpp:137-173): a snake_case name becomes
// CamelCase ("univariate_matern_stationary" -> "UnivariateMaternStationary"),
// the form the kernel registry and the parameter-count map are keyed by.
std::string camel_kernel_name(const std::string& v) {
  if (v.empty() || (v.find('_') == std::string::npos && !std::islower((unsigned char)v[0]))) return v;
  std::string out;
  bool up = true;
  for (char c : v) {
    if (c == '_') {
      up = true;
      continue;
    }
    out += up ? (char)std::toupper((unsigned char)c) : c;
    up = false;
  }
  return out;
}

// Validator::CheckDistanceMetricValue (Validator.cpp:285-294).  The likelihood
// path always evaluates Euclidean distances (ChameleonImplementation.cpp:172
// passes metric 0), here as in the reference; the value is kept for callers.
int parse_distance_metric(const std::string& v) {
  if (v == "eg" || v == "EG" || v == "euclidean") return common::EUCLIDEAN_DISTANCE;
  if (v == "gcd" || v == "GCD" || v == "great_circle") return common::GREAT_CIRCLE_DISTANCE;
  throw std::range_error("Invalid value. Please use eg or gcd values only.");
}

// Validator::CheckComputationValue (Validator.cpp:108-121): the same spellings
// and message; tile low-rank is a value the reference accepts but this build
// does not run.
common::Computation parse_computation(const std::string& v) {
  if (v == "exact" || v == "Exact" || v == "Dense" || v == "dense") return common::EXACT_DENSE;
  if (v == "diag_approx" || v == "diagonal_approx") return common::DIAGONAL_APPROX;
  if (v == "lr_approx" || v == "tlr" || v == "TLR")
    throw std::domain_error("--computation=" + v + ": tile low-rank is not on the B200 path");
  throw std::range_error("Invalid value for Computation. Please use Exact, diagonal_approx or TLR.");
}

// Validator::CheckPrecisionValue (Validator.cpp:123-136): the same spellings and
// message; single precision throughout is a value the reference accepts but
// this build does not run (its mixed form keeps FP64 where it matters).
common::Precision parse_precision(const std::string& v) {
  if (v == "double" || v == "Double") return common::DOUBLE;
  if (v == "mix" || v == "Mix" || v == "Mixed" || v == "mixed") return common::MIXED;
  if (v == "single" || v == "Single")
    throw std::domain_error("--precision=" + v + ": single precision is not on the B200 path");
  throw std::range_error("Invalid value for Computation. Please use Single, Double or Mixed.");
}

}  // namespace

void Configurations::InitializeArguments(const int& argc, char** argv) {
  for (int i = 1; i < argc; ++i) {
    std::string arg = argv[i];
    if (arg.rfind("--", 0) != 0) continue;
    arg = arg.substr(2);
    const size_t eq = arg.find('=');
    const std::string key = normalise_key(arg.substr(0, eq));
    const std::string val = eq == std::string::npos ? "true" : arg.substr(eq + 1);
    if (key == "n") SetProblemSize(std::stoi(val));
    else if (key == "kernel") SetKernelName(camel_kernel_name(val));
    else if (key == "dts") SetDenseTileSize(std::stoi(val));
    else if (key == "seed") SetSeed(std::stoi(val));
    else if (key == "maxmleiterations") SetMaxMleIterations(std::stoi(val));
    else if (key == "tolerance") SetTolerance(std::stod(val));
    else if (key == "zmiss") SetUnknownObservationsNb(std::stoi(val));
    else if (key == "itheta" || key == "initialtheta") SetInitialTheta(parse_theta(val));
    else if (key == "lb" || key == "lowerbounds") SetLowerBounds(parse_theta(val));
    else if (key == "ub" || key == "upperbounds") SetUpperBounds(parse_theta(val));
    else if (key == "etheta" || key == "estimatedtheta") SetEstimatedTheta(parse_theta(val));
    else if (key == "mspe") SetIsMSPE(parse_bool(val));
    else if (key == "fisher") SetIsFisher(parse_bool(val));
    else if (key == "mloemmom") SetIsMLOEMMOM(parse_bool(val));
    else if (key == "idw") {
      if (parse_bool(val)) throw std::domain_error("--idw: inverse-distance weighting is not on the B200 path");
      SetIsIDW(false);
    } else if (key == "isnongaussian") {
      if (parse_bool(val)) throw std::domain_error("--isnongaussian: non-Gaussian likelihoods are not on the B200 path");
      SetIsNonGaussian(false);
    } else if (key == "p" || key == "q") {
      // process grid of the reference's distributed runs; one process per GPU here
      if (std::stoi(val) != 1) throw std::domain_error("--" + key + "=" + val + ": one process drives one GPU here");
    } else if (key == "distancemetric") SetDistanceMetric(parse_distance_metric(val));
    else if (key == "observationnumber") SetObservationNumber(std::stoi(val));
    else if (key == "timeslot") SetTimeSlot(std::stoi(val));
    else if (key == "startingtheta") SetStartingTheta(parse_theta(val));
    else if (key == "lts") SetLowTileSize(std::stoi(val));
    else if (key == "maxrank") SetMaxRank(std::stoi(val));
    else if (key == "recoveryfile") SetRecoveryFile(val);
    else if (key == "computation") SetComputation(parse_computation(val));
    else if (key == "precision") SetPrecision(parse_precision(val));
    else if (key == "band") SetBand(std::stoi(val));
    else if (key == "mixedband") SetMixedPrecisionBand(std::stoi(val));  // this build: FP64 tile rows of --precision=mixed
    else if (key == "datapath") SetDataPath(val);
    else if (key == "dimension") {
      if (val != "2D" && val != "2d") throw std::domain_error("only 2D locations are on the B200 path");
      SetDimension(common::Dimension2D);
    } else if (key == "cores") SetCoresNumber(std::stoi(val));
    else if (key == "gpus") SetGPUsNumbers(std::stoi(val));
    else if (key == "verbose") SetVerbosity(val == "quiet" ? common::QUIET_MODE
                                            : val == "detailed" ? common::DETAILED_MODE : common::STANDARD_MODE);
    else throw std::invalid_argument("unknown or unsupported argument --" + arg);
  }
}

}  // namespace exageostat::configurations
