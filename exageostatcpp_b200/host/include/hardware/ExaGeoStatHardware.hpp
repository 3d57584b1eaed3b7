// Device initialisation (src/hardware/ExaGeoStatHardware.cpp:126-172 starts
// Chameleon/StarPU on `cores` CPU workers and `gpus` GPUs); here it selects
// CUDA device 0 and fails loudly when there is none -- there is no CPU path.
#pragma once
#include <stdexcept>
#include <string>
#include "common/Definitions.hpp"
#include "exageostat_b200.h"

class ExaGeoStatHardware {
 public:
  ExaGeoStatHardware(const exageostat::common::Computation& aComputation, const int& aCoreNumber,
                     const int& aGpuNumber, const int& aP = 1, const int& aQ = 1) {
    (void)aCoreNumber;
    (void)aGpuNumber;
    (void)aP;
    (void)aQ;
    if (aComputation == exageostat::common::TILE_LOW_RANK)
      throw std::domain_error("TILE_LOW_RANK (HiCMA) is not part of the B200 path");
    const int rc = egs_hardware_init(0);
    if (rc != EGS_OK)
      throw std::runtime_error(std::string("ExaGeoStatHardware: ") + egs_status_string(rc) + " " + egs_last_error());
  }
};
