// C++ API test driver: the reference's API-level tests (TestExaGeoStatApi.cpp,
// TestUnivariateMaternStationary.cpp, TestPrediction.cpp, TestSyntheticGenerator.cpp)
// re-expressed against the B200 host API.  Each case sets up Configurations the way
// the reference test does, runs the API, and prints one JSON line of results;
// tests/test_gpu_host_api.py compares them with the reference goldens.
//
// usage: test_exageostat_api <case> [fixture-file]
//   fixture-file: three lines of 16 numbers (x, y, z) -- the reference's N=16 fixture.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "api/ExaGeoStat.hpp"
#include "hardware/ExaGeoStatHardware.hpp"
#include "linear-algebra-solvers/LinearAlgebraFactory.hpp"

using namespace exageostat;
using namespace exageostat::common;
using namespace exageostat::configurations;
using namespace exageostat::dataunits;

namespace {

std::string json_array(const double* v, int n) {
  std::ostringstream os;
  os.precision(17);
  os << "[";
  for (int i = 0; i < n; ++i) os << (i ? "," : "") << v[i];
  os << "]";
  return os.str();
}

struct Fixture {
  std::vector<double> x, y, z;
};

Fixture read_fixture(const char* path) {
  Fixture f;
  std::ifstream in(path);
  std::vector<double>* rows[3] = {&f.x, &f.y, &f.z};
  std::string line;
  for (int r = 0; r < 3 && std::getline(in, line); ++r) {
    std::istringstream ls(line);
    double v;
    while (ls >> v) rows[r]->push_back(v);
  }
  if (f.x.size() != 16 || f.y.size() != 16 || f.z.size() != 16) throw std::runtime_error("bad fixture file");
  return f;
}

// TestExaGeoStatApi.cpp TEST_GENERATE_DATA / TestUnivariateMaternStationary.cpp
void generate(int n, int dts) {
  Configurations c;
  c.SetSeed(0);
  c.SetProblemSize(n);
  c.SetKernelName("UnivariateMaternStationary");
  c.SetDenseTileSize(dts);
  c.SetComputation(EXACT_DENSE);
  Configurations::SetVerbosity(QUIET_MODE);
  c.SetLowerBounds({0.1, 0.1, 0.1});
  c.SetUpperBounds({5, 5, 5});
  c.SetInitialTheta({1, 0.1, 0.5});
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 4, 0);
  std::unique_ptr<ExaGeoStatData<double>> data;
  api::ExaGeoStat<double>::ExaGeoStatLoadData(c, data);
  auto* A = (double*)data->GetDescriptorData()->GetDescriptor(CHAMELEON_DESCRIPTOR, DESCRIPTOR_Z).chameleon_desc->mat;
  std::cout << "{\"z\": " << json_array(A, n) << ", \"x\": " << json_array(data->GetLocations()->GetLocationX(), n)
            << ", \"y\": " << json_array(data->GetLocations()->GetLocationY(), n) << "}" << std::endl;
}

Configurations modeling_config() {
  Configurations c;
  c.SetSeed(0);
  c.SetProblemSize(16);
  c.SetKernelName("UnivariateMaternStationary");
  c.SetDenseTileSize(8);
  c.SetComputation(EXACT_DENSE);
  c.SetMaxMleIterations(3);
  c.SetTolerance(4);
  c.SetLowerBounds({0.1, 0.1, 0.1});
  c.SetStartingTheta({0.1, 0.1, 0.1});
  c.SetUpperBounds({5, 5, 5});
  c.SetInitialTheta({1, 0.1, 0.5});
  Configurations::SetVerbosity(QUIET_MODE);
  return c;
}

// TestExaGeoStatApi.cpp TEST_MODEL_DATA, section "Data Modeling", for the
// exact dense factorisation and the diagonal super-tile approximation (dts 8)
void modeling_fixture(const Fixture& f, Computation computation = EXACT_DENSE) {
  Configurations c = modeling_config();
  c.SetComputation(computation);
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 4, 0);
  auto data = std::make_unique<ExaGeoStatData<double>>(c.GetProblemSize(), c.GetDimension());
  std::vector<double> z = f.z, x = f.x, y = f.y;
  data->GetLocations()->SetLocationX(*x.data(), 16);
  data->GetLocations()->SetLocationY(*y.data(), 16);
  double ll = api::ExaGeoStat<double>::ExaGeoStatDataModeling(c, data, z.data());
  std::cout.precision(17);
  std::cout << "{\"loglik\": " << ll << ", \"theta\": " << json_array(c.GetEstimatedTheta().data(), 3)
            << ", \"iterations\": " << data->GetMleIterations() << "}" << std::endl;
}

// TestExaGeoStatApi.cpp TEST_MODEL_DATA, section "Data Generation and Modeling"
void generate_and_model() {
  Configurations c = modeling_config();
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 4, 0);
  std::unique_ptr<ExaGeoStatData<double>> data;
  api::ExaGeoStat<double>::ExaGeoStatLoadData(c, data);
  double ll = api::ExaGeoStat<double>::ExaGeoStatDataModeling(c, data);
  std::cout.precision(17);
  std::cout << "{\"loglik\": " << ll << ", \"theta\": " << json_array(c.GetEstimatedTheta().data(), 3) << "}"
            << std::endl;
}

// --precision=mixed through the API: the same synthetic data modelled with
// three BOBYQA evaluations in FP64 and in mixed precision (FP64 band of 2 tiles).
void mixed_modeling() {
  Configurations c = modeling_config();
  c.SetProblemSize(3000);
  c.SetDenseTileSize(256);
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 4, 0);
  std::unique_ptr<ExaGeoStatData<double>> data;
  api::ExaGeoStat<double>::ExaGeoStatLoadData(c, data);
  const double ll_double = api::ExaGeoStat<double>::ExaGeoStatDataModeling(c, data);
  const std::vector<double> th_double = c.GetEstimatedTheta();
  c.SetPrecision(MIXED);
  c.SetStartingTheta({0.1, 0.1, 0.1});
  data->SetMleIterations(0);
  const double ll_mixed = api::ExaGeoStat<double>::ExaGeoStatDataModeling(c, data);
  std::cout.precision(17);
  std::cout << "{\"loglik_double\": " << ll_double << ", \"loglik_mixed\": " << ll_mixed
            << ", \"theta_double\": " << json_array(th_double.data(), 3)
            << ", \"theta_mixed\": " << json_array(c.GetEstimatedTheta().data(), 3) << "}" << std::endl;
}

// TestPrediction.cpp TEST_PREDICTION_MISSING_DATA, section "Test Prediction - MSPE"
void prediction_mspe(const Fixture& f) {
  Configurations c;
  c.SetUnknownObservationsNb(4);
  c.SetProblemSize(16);
  c.SetKernelName("UnivariateMaternStationary");
  c.SetDenseTileSize(8);
  c.SetComputation(EXACT_DENSE);
  c.SetMaxMleIterations(3);
  c.SetTolerance(4);
  c.SetLowerBounds({0.1, 0.1, 0.1});
  c.SetStartingTheta({0.1, 0.1, 0.1});
  c.SetUpperBounds({5, 5, 5});
  c.SetInitialTheta({1, 0.1, 0.5});
  Configurations::SetVerbosity(QUIET_MODE);
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, c.GetCoresNumber(), c.GetGPUsNumbers());
  auto data = std::make_unique<ExaGeoStatData<double>>(c.GetProblemSize(), c.GetDimension());
  std::vector<double> z = f.z, x = f.x, y = f.y;
  data->GetLocations()->SetLocationX(*x.data(), 16);
  data->GetLocations()->SetLocationY(*y.data(), 16);
  c.SetIsMSPE(true);
  c.SetEstimatedTheta({0.9, 0.09, 0.4});
  kernels::Kernel<double>* pKernel =
      plugins::PluginRegistry<kernels::Kernel<double>>::Create(c.GetKernelName(), c.GetTimeSlot());
  prediction::Prediction<double>::PredictMissingData(data, c, z.data(), *pKernel);
  delete pKernel;
  auto zm = results::Results::GetInstance()->GetPredictedMissedValues();
  std::cout.precision(17);
  std::cout << "{\"mspe\": " << results::Results::GetInstance()->GetMSPEError()
            << ", \"z_miss\": " << json_array(zm.data(), (int)zm.size()) << "}" << std::endl;
}

// TestSyntheticGenerator.cpp TEST_GENERATION
void generated_locations() {
  Configurations c;
  c.SetDimension(Dimension2D);
  c.SetInitialTheta({1, 0.1, 0.5});
  c.SetProblemSize(9);
  c.SetDenseTileSize(1);
  c.SetKernelName("UnivariateMaternStationary");
  c.SetComputation(EXACT_DENSE);
  srand(0);
  Locations<double> l(9, Dimension2D);
  generators::SyntheticGenerator<double>::GenerateLocations(9, l);
  Locations<double> l1(9, Dimension2D);
  generators::SyntheticGenerator<double>::GenerateLocations(9, l1);  // continues the rand() sequence
  srand(0);
  Locations<double> l2(9, Dimension2D);
  generators::SyntheticGenerator<double>::GenerateLocations(9, l2);
  std::cout << "{\"x\": " << json_array(l.GetLocationX(), 9) << ", \"y\": " << json_array(l.GetLocationY(), 9)
            << ", \"x_second\": " << json_array(l1.GetLocationX(), 9)
            << ", \"x_reseeded\": " << json_array(l2.GetLocationX(), 9) << "}" << std::endl;
}

// Kernel plugin on the host interface, and the reference's error behaviour.
void plugin_and_errors(const Fixture& f) {
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 1, 1);
  Locations<double> l(16, Dimension2D);
  std::vector<double> x = f.x, y = f.y;
  l.SetLocationX(*x.data(), 16);
  l.SetLocationY(*y.data(), 16);
  kernels::Kernel<double>* k =
      plugins::PluginRegistry<kernels::Kernel<double>>::Create("UnivariateMaternStationary", 1);
  double theta[3] = {1.3, 0.2, 0.5};
  std::vector<double> a(5 * 7);
  k->GenerateCovarianceMatrix(a.data(), 5, 7, 3, 6, l, l, l, theta, 0);
  double maxerr = 0;
  for (int j = 0; j < 7; ++j)
    for (int i = 0; i < 5; ++i) {
      const double dx = x[6 + j] - x[3 + i], dy = y[6 + j] - y[3 + i];
      const double d = std::sqrt(dx * dx + dy * dy) / 0.2;
      const double ref = d == 0 ? 1.3 : 1.3 * std::exp(-d);
      maxerr = std::max(maxerr, std::fabs(a[i + j * 5] - ref) / std::fabs(ref));
    }
  delete k;
  std::string unknown_kernel, non_spd, no_theta;
  try {
    plugins::PluginRegistry<kernels::Kernel<double>>::Create("NoSuchKernel", 1);
  } catch (const std::exception& e) {
    unknown_kernel = e.what();
  }
  try {
    Configurations c = modeling_config();
    auto data = std::make_unique<ExaGeoStatData<double>>(16, Dimension2D);
    std::vector<double> xs = f.x, ys = f.y, z = f.z;
    xs[5] = std::nan("");
    data->GetLocations()->SetLocationX(*xs.data(), 16);
    data->GetLocations()->SetLocationY(*ys.data(), 16);
    api::ExaGeoStat<double>::ExaGeoStatDataModeling(c, data, z.data());
  } catch (const std::exception& e) {
    non_spd = e.what();
  }
  try {
    Configurations c = modeling_config();
    c.SetIsMSPE(true);
    c.SetUnknownObservationsNb(4);
    auto data = std::make_unique<ExaGeoStatData<double>>(16, Dimension2D);
    std::vector<double> z = f.z;
    kernels::Kernel<double>* kk =
        plugins::PluginRegistry<kernels::Kernel<double>>::Create("UnivariateMaternStationary", 1);
    std::unique_ptr<kernels::Kernel<double>> guard(kk);
    c.InitializeAllTheta();
    prediction::Prediction<double>::PredictMissingData(data, c, z.data(), *kk);
  } catch (const std::exception& e) {
    no_theta = e.what();
  }
  std::cout.precision(17);
  std::cout << "{\"plugin_max_rel_err\": " << maxerr << ", \"unknown_kernel\": \"" << unknown_kernel
            << "\", \"non_spd\": \"" << non_spd << "\", \"no_theta\": \"" << no_theta.substr(0, 40) << "\"}"
            << std::endl;
}

}  // namespace


// TestPrediction.cpp sections "MLOE_MMOM" and "FISHER": the reference's Catch test
// re-runs its body per SECTION in one process, so the MLOE/MMOM section draws the
// third hold-out split (after the MSPE and IDW sections); the same sequence here.
void prediction_aux(const Fixture& f) {
  Configurations c;
  c.SetUnknownObservationsNb(4);
  c.SetProblemSize(16);
  c.SetKernelName("UnivariateMaternStationary");
  c.SetDenseTileSize(8);
  c.SetComputation(EXACT_DENSE);
  c.SetInitialTheta({1, 0.1, 0.5});
  c.SetEstimatedTheta({0.9, 0.09, 0.4});
  Configurations::SetVerbosity(QUIET_MODE);
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, c.GetCoresNumber(), c.GetGPUsNumbers());
  kernels::Kernel<double>* pKernel =
      plugins::PluginRegistry<kernels::Kernel<double>>::Create(c.GetKernelName(), c.GetTimeSlot());
  auto run = [&](bool mspe, bool mloe, bool fisher) {
    auto data = std::make_unique<ExaGeoStatData<double>>(c.GetProblemSize(), c.GetDimension());
    std::vector<double> z = f.z, x = f.x, y = f.y;
    data->GetLocations()->SetLocationX(*x.data(), 16);
    data->GetLocations()->SetLocationY(*y.data(), 16);
    c.SetIsMSPE(mspe);
    c.SetIsMLOEMMOM(mloe);
    c.SetIsFisher(fisher);
    prediction::Prediction<double>::PredictMissingData(data, c, z.data(), *pKernel);
  };
  run(true, false, false);   // the MSPE section
  run(true, false, false);   // the IDW section's split
  run(false, true, false);   // MLOE / MMOM
  auto* r = results::Results::GetInstance();
  const double mloe = r->GetMLOE(), mmom = r->GetMMOM();
  run(false, false, true);   // Fisher (no split needed)
  auto fisher = r->GetFisherMatrix();
  delete pKernel;
  std::cout.precision(17);
  std::cout << "{\"mloe\": " << mloe << ", \"mmom\": " << mmom << ", \"fisher\": "
            << json_array(fisher.data(), (int)fisher.size()) << "}" << std::endl;
}


// CSV round trip: synthetic data written by the CSV writer, read back by the
// loader through ExaGeoStatLoadData (--datapath), then modelled.
void csv_roundtrip(const std::string& dir) {
  Configurations c = modeling_config();
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 4, 0);
  std::unique_ptr<ExaGeoStatData<double>> gen;
  api::ExaGeoStat<double>::ExaGeoStatLoadData(c, gen);
  std::vector<double> z = gen->GetDescriptorData()->HostVector(DESCRIPTOR_Z);
  const std::string file =
      dataLoader::csv::CSVLoader<double>::WriteData(z.data(), 16, dir, *gen->GetLocations());
  Configurations c2 = modeling_config();
  c2.SetProblemSize(0);
  c2.SetDataPath(file);
  std::unique_ptr<ExaGeoStatData<double>> loaded;
  api::ExaGeoStat<double>::ExaGeoStatLoadData(c2, loaded);
  double dmax = 0;
  std::vector<double>& z2 = loaded->GetDescriptorData()->HostVector(DESCRIPTOR_Z);
  for (int i = 0; i < 16; ++i) {
    dmax = std::max(dmax, std::fabs(z2[i] - z[i]));
    dmax = std::max(dmax, std::fabs(loaded->GetLocations()->GetLocationX()[i] - gen->GetLocations()->GetLocationX()[i]));
    dmax = std::max(dmax, std::fabs(loaded->GetLocations()->GetLocationY()[i] - gen->GetLocations()->GetLocationY()[i]));
  }
  const double ll_gen = api::ExaGeoStat<double>::ExaGeoStatDataModeling(c, gen);
  const double ll_csv = api::ExaGeoStat<double>::ExaGeoStatDataModeling(c2, loaded);
  std::string bad = "none";
  {
    std::ofstream o(dir + "/bad.csv");
    o << "0.1,0.2,0.3,0.4\n";
  }
  Configurations c3 = modeling_config();
  c3.SetDataPath(dir + "/bad.csv");
  try {
    std::unique_ptr<ExaGeoStatData<double>> d3;
    api::ExaGeoStat<double>::ExaGeoStatLoadData(c3, d3);
  } catch (const std::exception& e) {
    bad = e.what();
  }
  std::cout.precision(17);
  std::cout << "{\"n\": " << c2.GetProblemSize() << ", \"max_diff\": " << dmax << ", \"loglik_generated\": " << ll_gen
            << ", \"loglik_csv\": " << ll_csv << ", \"bad\": \"" << bad << "\"}" << std::endl;
}

// The seam's tile operations (LinearAlgebraMethods.hpp:62-64, 153-216, 275, 286)
// driven the way ChameleonImplementation<T>::ExaGeoStatMLETile strings them
// together (ChameleonImplementation.cpp:113-265), on descriptor handles from
// DescriptorData::GetDescriptor: the log-likelihood assembled from the factor's
// diagonal and the solved Z must equal one egs_mle_eval; dposv, the copies
// between LAPACK and descriptor layouts and the argument checks are exercised too.
void seam_tile_operations() {
  Configurations c = modeling_config();
  c.SetProblemSize(700);
  c.SetDenseTileSize(128);
  const std::vector<double> theta = {1.0, 0.1, 0.5};
  auto hardware = ExaGeoStatHardware(EXACT_DENSE, 4, 0);
  std::unique_ptr<ExaGeoStatData<double>> data;
  api::ExaGeoStat<double>::ExaGeoStatLoadData(c, data);
  const int n = c.GetProblemSize();
  std::vector<double> z = data->GetDescriptorData()->HostVector(DESCRIPTOR_Z);
  auto solver = linearAlgebra::LinearAlgebraFactory<double>::CreateLinearAlgebraSolver(EXACT_DENSE);
  DescriptorData<double> dd;
  solver->InitiateDescriptors(c, dd, 1, z.data());
  egs_problem* p = dd.GetProblem();
  EgsCheck(egs_problem_set_locations(p, data->GetLocations()->GetLocationX(), data->GetLocations()->GetLocationY()),
           "egs_problem_set_locations");
  void* C = dd.GetDescriptor(CHAMELEON_DESCRIPTOR, DESCRIPTOR_C).chameleon_desc;
  void* Z = dd.GetDescriptor(CHAMELEON_DESCRIPTOR, DESCRIPTOR_Z).chameleon_desc;
  void* Zcpy = dd.GetDescriptor(CHAMELEON_DESCRIPTOR, DESCRIPTOR_Z_COPY).chameleon_desc;
  void* sequence = nullptr;
  solver->ExaGeoStatCreateSequence(&sequence);
  EgsCheck(egs_problem_set_stream(p, sequence), "egs_problem_set_stream");
  solver->ExaGeoStatLapackCopyTile(EXAGEOSTAT_UPPER_LOWER, Z, Zcpy);
  EgsCheck(egs_covariance_generate(p, theta.data()), "egs_covariance_generate");
  std::vector<double> cov((size_t)n * n, 0.0), cov_back((size_t)n * n, 0.0);
  solver->ExaGeoStatDesc2Lap(cov.data(), n, C, EXAGEOSTAT_LOWER);
  solver->ExaGeoStatPotrfTile(EXAGEOSTAT_LOWER, C, 0, nullptr, nullptr, 0, 0);
  std::vector<double> factor((size_t)n * n, 0.0);
  solver->ExaGeoStatDesc2Lap(factor.data(), n, C, EXAGEOSTAT_LOWER);
  solver->ExaGeoStatTrsmTile(EXAGEOSTAT_LEFT, EXAGEOSTAT_LOWER, EXAGEOSTAT_NO_TRANS, EXAGEOSTAT_NON_UNIT, 1.0, C,
                             nullptr, nullptr, Z, 0);
  solver->ExaGeoStatSequenceWait(sequence);
  std::vector<double> v(n);
  solver->ExaGeoStatDesc2Lap(v.data(), n, Z, EXAGEOSTAT_UPPER_LOWER);
  double logdet = 0, dot = 0;
  for (int i = 0; i < n; ++i) {
    logdet += 2.0 * std::log(factor[i + (size_t)i * n]);
    dot += v[i] * v[i];
  }
  const double ll_tiles = -0.5 * dot - 0.5 * logdet - (n / 2.0) * std::log(2.0 * PI);
  // dposv on the regenerated covariance, restored Z: w = C^-1 z
  solver->ExaGeoStatLapackCopyTile(EXAGEOSTAT_UPPER_LOWER, Zcpy, Z);
  solver->ExaGeoStatLap2Desc(cov.data(), n, C, EXAGEOSTAT_LOWER);
  std::vector<double> cov_uploaded((size_t)n * n, 0.0);
  solver->ExaGeoStatDesc2Lap(cov_uploaded.data(), n, C, EXAGEOSTAT_LOWER);
  double roundtrip = 0;
  for (size_t i = 0; i < cov.size(); ++i) roundtrip = std::max(roundtrip, std::fabs(cov[i] - cov_uploaded[i]));
  solver->ExaGeoStatPosvTile(EXAGEOSTAT_LOWER, C, Z);
  std::vector<double> w(n);
  solver->ExaGeoStatDesc2Lap(w.data(), n, Z, EXAGEOSTAT_LOWER);
  // the same evaluation in one call
  solver->ExaGeoStatLapackCopyTile(EXAGEOSTAT_UPPER_LOWER, Zcpy, Z);
  double ll_eval = 0;
  EgsCheck(egs_mle_eval(p, theta.data(), &ll_eval, nullptr, nullptr), "egs_mle_eval");
  // the forms the device does not take are refused with the reference's exception types
  std::string bad_uplo = "none", bad_trans = "none", bad_desc = "none";
  try {
    solver->ExaGeoStatPotrfTile(EXAGEOSTAT_UPPER, C, 0, nullptr, nullptr, 0, 0);
  } catch (const std::domain_error& e) {
    bad_uplo = e.what();
  }
  try {
    solver->ExaGeoStatTrsmTile(EXAGEOSTAT_RIGHT, EXAGEOSTAT_LOWER, EXAGEOSTAT_NO_TRANS, EXAGEOSTAT_NON_UNIT, 1.0, C,
                               nullptr, nullptr, Z, 0);
  } catch (const std::domain_error& e) {
    bad_trans = e.what();
  }
  try {
    solver->ExaGeoStatPotrfTile(EXAGEOSTAT_LOWER, Z, 0, nullptr, nullptr, 0, 0);
  } catch (const std::domain_error& e) {
    bad_desc = e.what();
  }
  EgsCheck(egs_problem_set_stream(p, nullptr), "egs_problem_set_stream");
  EgsCheck(egs_sequence_destroy(sequence), "egs_sequence_destroy");
  std::cout.precision(17);
  std::cout << "{\"n\": " << n << ", \"loglik_tiles\": " << ll_tiles << ", \"loglik_eval\": " << ll_eval
            << ", \"logdet\": " << logdet << ", \"dot\": " << dot << ", \"roundtrip\": " << roundtrip
            << ", \"w\": " << json_array(w.data(), n) << ", \"z\": " << json_array(z.data(), n)
            << ", \"x\": " << json_array(data->GetLocations()->GetLocationX(), n)
            << ", \"y\": " << json_array(data->GetLocations()->GetLocationY(), n) << ", \"bad_uplo\": \"" << bad_uplo
            << "\", \"bad_trans\": \"" << bad_trans << "\", \"bad_desc\": \"" << bad_desc << "\"}" << std::endl;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: test_exageostat_api <case> [fixture-file]\n";
    return 2;
  }
  const std::string which = argv[1];
  try {
    if (which == "generate_n16") generate(16, 9);
    else if (which == "generate_n9") generate(9, 5);
    else if (which == "modeling_fixture") modeling_fixture(read_fixture(argv[2]));
    else if (which == "modeling_fixture_dst") modeling_fixture(read_fixture(argv[2]), DIAGONAL_APPROX);
    else if (which == "generate_and_model") generate_and_model();
    else if (which == "mixed_modeling") mixed_modeling();
    else if (which == "prediction_mspe") prediction_mspe(read_fixture(argv[2]));
    else if (which == "prediction_aux") prediction_aux(read_fixture(argv[2]));
    else if (which == "csv_roundtrip") csv_roundtrip(argv[2]);
    else if (which == "generated_locations") generated_locations();
    else if (which == "plugin_and_errors") plugin_and_errors(read_fixture(argv[2]));
    else if (which == "seam_tile_operations") seam_tile_operations();
    else {
      std::cerr << "unknown case " << which << "\n";
      return 2;
    }
  } catch (const std::exception& e) {
    std::cerr << "exception: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
