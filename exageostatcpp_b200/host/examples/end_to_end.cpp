// End-to-end run of the ExaGeoStat<T> API on one B200, driven by the same
// command-line flags as the reference's examples (examples/end-to-end/
// DataGenerationModelingAndPrediction.cpp): generate (or, with --datapath, load)
// the data, fit theta by maximum likelihood, then predict --zmiss held-out
// values with MSPE, and the Fisher matrix and MLOE/MMOM when asked for.
//
//   end_to_end --N=1600 --dts=320 --kernel=univariate_matern_stationary \
//       --itheta=1:0.1:0.5 --lb=0.1:0.01:0.01 --ub=5:5:5 --tolerance=4 \
//       --max_mle_iterations=20 --zmiss=10 --mspe=true [--precision=mixed]
//
// Without a CUDA device it stops with the library's error (there is no CPU path).
#include <cstdio>
#include <exception>
#include <memory>

#include "api/ExaGeoStat.hpp"
#include "hardware/ExaGeoStatHardware.hpp"
#include "results/Results.hpp"

using exageostat::api::ExaGeoStat;
using exageostat::configurations::Configurations;
using exageostat::dataunits::ExaGeoStatData;
using exageostat::results::Results;

int main(int argc, char** argv) {
  try {
    Configurations configurations;
    configurations.InitializeArguments(argc, argv);
    ExaGeoStatHardware hardware(configurations.GetComputation(), configurations.GetCoresNumber(),
                                configurations.GetGPUsNumbers());
    std::unique_ptr<ExaGeoStatData<double>> data;
    ExaGeoStat<double>::ExaGeoStatLoadData(configurations, data);
    ExaGeoStat<double>::ExaGeoStatDataModeling(configurations, data);
    const bool predict = configurations.GetUnknownObservationsNb() > 0 &&
                         (configurations.GetIsMSPE() || configurations.GetIsFisher() ||
                          configurations.GetIsMLOEMMOM());
    if (predict) ExaGeoStat<double>::ExaGeoStatPrediction(configurations, data);

    const Results* r = Results::GetInstance();
    std::printf("N %d, precision %s\n", configurations.GetProblemSize(),
                configurations.GetPrecision() == exageostat::common::MIXED ? "mixed" : "double");
    std::printf("log-likelihood %.10f after %d evaluations\n", r->GetLogLikValue(), r->GetMLEIterations());
    const auto theta = r->GetMaximumTheta();
    std::printf("theta");
    for (double t : theta) std::printf(" %.8f", t);
    std::printf("\n");
    if (predict && configurations.GetIsMSPE()) std::printf("MSPE %.10f\n", r->GetMSPEError());
    if (predict && configurations.GetIsMLOEMMOM()) std::printf("MLOE %.10f MMOM %.10f\n", r->GetMLOE(), r->GetMMOM());
    if (predict && configurations.GetIsFisher()) {
      const auto f = r->GetFisherMatrix();
      std::printf("Fisher inverse");
      for (double v : f) std::printf(" %.6e", v);
      std::printf("\n");
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "end_to_end: %s\n", e.what());
    return 1;
  }
}
