// Host-only checks of the command-line parser of Configurations
// (exageostatcpp_b200/host/src/Configurations.cpp, following the reference's
// Parser.cpp:23-81 and Validator.cpp:108-173, 285-294): accepted spellings, the values
// they set, and the errors for values the reference rejects or this build does
// not run.  No GPU call is made.  Prints one "name: ok|FAIL ..." line per case
// and exits non-zero if any case failed.
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>
#include "configurations/Configurations.hpp"

using exageostat::configurations::Configurations;
namespace common = exageostat::common;

namespace {

int failures = 0;

void report(const char* name, bool ok, const std::string& why = "") {
  std::printf("%s: %s%s%s\n", name, ok ? "ok" : "FAIL", why.empty() ? "" : " ", why.c_str());
  if (!ok) ++failures;
}

void parse(Configurations& c, std::vector<std::string> args) {
  args.insert(args.begin(), "prog");
  std::vector<char*> argv;
  for (auto& a : args) argv.push_back(a.data());
  c.InitializeArguments((int)argv.size(), argv.data());
}

// "kind:message" of the exception parsing `args` throws, or "" if none.
std::string parse_error(std::vector<std::string> args) {
  Configurations c;
  try {
    parse(c, std::move(args));
  } catch (const std::domain_error& e) {
    return std::string("domain:") + e.what();
  } catch (const std::range_error& e) {
    return std::string("range:") + e.what();
  } catch (const std::invalid_argument& e) {
    return std::string("invalid:") + e.what();
  } catch (const std::exception& e) {
    return std::string("other:") + e.what();
  }
  return "";
}

}  // namespace

int main() {
  {
    Configurations c;
    parse(c, {"--N=1600", "--dts=320", "--kernel=univariate_matern_stationary", "--precision=mixed",
              "--mixedband=3", "--datapath=/tmp/data.csv", "--computation=exact", "--lb=0.1:0.1:0.1",
              "--ub=5:5:5", "--tolerance=9", "--max_mle_iterations=100"});
    report("mixed_run", c.GetProblemSize() == 1600 && c.GetDenseTileSize() == 320 &&
                            c.GetKernelName() == "UnivariateMaternStationary" &&
                            c.GetPrecision() == common::MIXED && c.GetMixedPrecisionBand() == 3 &&
                            c.GetDataPath() == "/tmp/data.csv" && c.GetComputation() == common::EXACT_DENSE &&
                            c.GetLowerBounds().size() == 3 && c.GetLowerBounds()[1] == 0.1 &&
                            c.GetUpperBounds()[2] == 5.0 && c.GetMaxMleIterations() == 100);
  }
  {
    Configurations c;
    parse(c, {"--computation=diag_approx", "--band=2"});
    report("diag_approx", c.GetComputation() == common::DIAGONAL_APPROX && c.GetBand() == 2);
    Configurations d;
    parse(d, {"--computation=Dense", "--precision=Double", "--kernel=UnivariateMaternStationary"});
    report("dense_double", d.GetComputation() == common::EXACT_DENSE && d.GetPrecision() == common::DOUBLE &&
                               d.GetKernelName() == "UnivariateMaternStationary");
    Configurations e;
    parse(e, {"--precision=mix", "--computation=diagonal_approx"});
    report("mix_spelling", e.GetPrecision() == common::MIXED && e.GetComputation() == common::DIAGONAL_APPROX);
  }
  {
    const std::string a = parse_error({"--precision=quad"});
    report("precision_invalid", a == "range:Invalid value for Computation. Please use Single, Double or Mixed.", a);
    const std::string b = parse_error({"--precision=single"});
    report("precision_single_not_run", b.rfind("domain:", 0) == 0, b);
    const std::string c = parse_error({"--computation=foo"});
    report("computation_invalid", c == "range:Invalid value for Computation. Please use Exact, diagonal_approx or TLR.",
           c);
    const std::string d = parse_error({"--computation=tlr"});
    report("computation_tlr_not_run", d.rfind("domain:", 0) == 0, d);
    const std::string e = parse_error({"--no_such_option=1"});
    report("unknown_argument", e.rfind("invalid:", 0) == 0, e);
    const std::string f = parse_error({"--dimension=3D"});
    report("dimension_3d_not_run", f.rfind("domain:", 0) == 0, f);
    const std::string g = parse_error({"--distance_metric=manhattan"});
    report("distance_invalid", g == "range:Invalid value. Please use eg or gcd values only.", g);
    const std::string h = parse_error({"--idw=true"});
    report("idw_not_run", h.rfind("domain:", 0) == 0, h);
    const std::string i = parse_error({"--p=2"});
    report("process_grid_not_run", i.rfind("domain:", 0) == 0, i);
  }
  {
    Configurations c;
    parse(c, {"--fisher=true", "--mloe_mmom=true", "--mspe=true", "--distance_metric=gcd", "--p=1", "--q=1",
              "--observation_number=4", "--idw=false", "--starting_theta=1:0.1:0.5"});
    report("prediction_flags", c.GetIsFisher() && c.GetIsMLOEMMOM() && c.GetIsMSPE() && !c.GetIsIDW() &&
                                   c.GetDistanceMetric() == common::GREAT_CIRCLE_DISTANCE &&
                                   c.GetObservationNumber() == 4 && c.GetStartingTheta().size() == 3 &&
                                   c.GetStartingTheta()[2] == 0.5);
  }
  return failures == 0 ? 0 : 1;
}
