// dispatch.h -- stage dispatch to the GPU (restates src/dispatch/mod.rs and
// src/dispatch/gpu.rs on top of the C ABI of include/drift_b200.h).
#pragma once

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "model.h"

namespace drift_host {

// drift.DriftError / drift.IntegrationError (src/interface/error.rs:13-46).
struct DriftErrorCpp : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct IntegrationErrorCpp : DriftErrorCpp {
    using DriftErrorCpp::DriftErrorCpp;
};

[[noreturn]] void raise_not_implemented(const std::string &msg);

// Python logging bridge: records carry the logger name, level, message and
// the C++ source position; a handler that raises is reported through
// sys.unraisablehook and does not abort the integration
// (src/logging.rs:10-53).
void log_record(const char *logger, int level, const char *file, int line, const std::string &msg);
constexpr int LOG_DEBUG = 10;
constexpr int LOG_INFO = 20;

struct StageStats {
    pybind11::array_t<uint32_t> accepted;
    pybind11::array_t<uint32_t> rejected;
    pybind11::array_t<uint8_t> status;
    double seconds = 0.0;        // the stage's wall time, copies included
    uint64_t bytes_in = 0;       // initial states and grid copied to the device
    uint64_t bytes_written = 0;  // trajectory bytes the stage produced
};

// Integrates every stage of `plan`; result[i] is the (nt, N, 6) trajectory
// of plan.stages[i]: a numpy array, or with `device_out` a torch CUDA tensor
// written in place by the kernels (no host round trip).  `stats`, if
// non-null, receives per-stage counters.
std::vector<pybind11::object> gpu_dispatch(const Config &config, const IntegrationPlan &plan,
                                           std::vector<StageStats> *stats, bool device_out = false);

}  // namespace drift_host
