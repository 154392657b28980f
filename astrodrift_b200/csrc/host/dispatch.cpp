// dispatch.cpp -- stage dispatch to the GPU through the C ABI.
//
// Restates gpu_dispatch / launch_kernel / dispatch_stages
// (src/dispatch/gpu.rs:157-229, src/dispatch/mod.rs:14-34): log the request,
// integrate each state-bearing stage in dependency order, return time-major
// (nt, N, 6) trajectories.  Differences from the reference, by design:
//  * the stage force comes from the model (the reference ignores the model
//    and always integrates a unit Kepler mass, src/dispatch/gpu.rs:155-156):
//    the sum of every stationary background the stage requires and, with
//    Config(attached_potentials=True), of the potentials attached to the
//    particle groups it requires, which move along those groups'
//    trajectories from their own, earlier stages;
//  * per-particle failures (galpy's DOPR54 error code, step cap, timeout)
//    raise IntegrationError, as the reference's CPU path does for DOPR54
//    (src/dispatch/cpu.rs:35-38, src/dispatch/mod.rs:74-75);
//  * the GIL is released while the device works.
#include "dispatch.h"

#include <chrono>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "drift_b200.h"

namespace py = pybind11;
using namespace pybind11::literals;

namespace drift_host {

namespace {

const char *LOG_GPU = "drift.dispatch.gpu";
const char *LOG_BACKEND = "drift.dispatch.gpu.b200";

std::string fmt(const char *f, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof(buf), f, ap);
    va_end(ap);
    return buf;
}

// Rust's `{}` for f64: shortest text that round-trips, integers without ".0".
std::string rust_float(double v)
{
    if (std::isfinite(v) && v == std::floor(v) && std::fabs(v) < 1e16) return fmt("%.0f", v);
    for (int p = 1; p <= 17; p++) {
        std::string s = fmt("%.*g", p, v);
        if (std::strtod(s.c_str(), nullptr) == v) return s;
    }
    return fmt("%.17g", v);
}

// Rust's `{:.3?}` for a Duration.
std::string rust_duration(double seconds)
{
    if (seconds >= 1.0) return fmt("%.3fs", seconds);
    if (seconds >= 1e-3) return fmt("%.3fms", seconds * 1e3);
    if (seconds >= 1e-6) return fmt("%.3fus", seconds * 1e6);
    return fmt("%.3fns", seconds * 1e9);
}

drift_potential potential_of(const Recipe &r)
{
    drift_potential p;
    std::memset(&p, 0, sizeof(p));
    switch (r.name) {
    case PotentialName::Kepler:
    case PotentialName::CustomKepler:
        p.kind = DRIFT_POT_KEPLER;
        p.amp = r.amp;
        break;
    case PotentialName::Plummer:
    case PotentialName::CustomPlummer:
        p.kind = DRIFT_POT_PLUMMER;
        p.amp = r.amp;
        p.b = r.radius;
        break;
    case PotentialName::Bovy:
        if (drift_potential_bovy(&p, r.bulge_alpha, r.bulge_rc, r.bulge_force, r.mn_amp, r.mn_a,
                                 r.mn_b, r.nfw_amp, r.nfw_a) != DRIFT_SUCCESS)
            throw py::value_error(std::string("invalid Bovy parameters: ") + drift_last_error());
        break;
    }
    return p;
}

const char *status_name(int s)
{
    switch (s) {
    case DRIFT_PARTICLE_MIN_STEP: return "minimum step reached";
    case DRIFT_PARTICLE_MAX_STEPS: return "step limit reached";
    case DRIFT_PARTICLE_NONFINITE: return "non-finite error estimate";
    case DRIFT_PARTICLE_TIMEOUT: return "device time budget exhausted";
    default: return "ok";
    }
}

// The force a stage integrates in: one stationary potential (the direct
// path), or a drift_force_model with its origin table on the host.
struct StageForce {
    bool single = false;
    drift_potential pot{};
    drift_force_model model{};
    std::vector<double> origins;  // host table (n_segments, n_sources, 18)
    py::object origins_dev;       // device table (run(device=True))
    // The force as a model (for the accelerations of this stage's particles
    // when a later stage uses them as moving sources); model.origins points
    // at the table of the current mode.
    drift_force_model as_model() const
    {
        if (!single) return model;
        drift_force_model m{};
        m.n_static = 1;
        m.statics[0] = pot;
        return m;
    }
};

drift_source_group source_group_of(const Recipe &r)
{
    drift_source_group g{};
    g.kind = r.name == PotentialName::CustomPlummer ? DRIFT_POT_PLUMMER : DRIFT_POT_KEPLER_CARTESIAN;
    g.amp = r.amp;
    g.b = r.radius;
    return g;
}

}  // namespace

[[noreturn]] void raise_not_implemented(const std::string &msg)
{
    PyErr_SetString(PyExc_NotImplementedError, msg.c_str());
    throw py::error_already_set();
}

void log_record(const char *logger_name, int level, const char *file, int line, const std::string &msg)
{
    py::object logging = py::module_::import("logging");
    py::object logger = logging.attr("getLogger")(logger_name);
    if (!logger.attr("isEnabledFor")(level).cast<bool>()) return;
    try {
        py::object rec = logger.attr("makeRecord")(logger_name, level, file, line, msg, py::tuple(),
                                                   py::none());
        logger.attr("handle")(rec);
    } catch (py::error_already_set &e) {
        e.discard_as_unraisable(py::str("drift logging handler"));
    }
}

#define DRIFT_LOG(logger, level, msg) log_record(logger, level, "gpu_dispatch.cpp", __LINE__, msg)

std::vector<py::object> gpu_dispatch(const Config &config, const IntegrationPlan &plan,
                                     std::vector<StageStats> *stats, bool device_out)
{
    const OutputGrid &ts = config.output;
    DRIFT_LOG(LOG_GPU, LOG_INFO,
              fmt("GPU integration starting: implementation=%s, method=%s, %lld output times over [%s, %s], rtol=%.2e, atol=%.2e",
                  name_of(config.implementation), name_of(config.method), (long long)ts.steps,
                  rust_float(ts.start).c_str(), rust_float(ts.end).c_str(), config.tolerance.rtol,
                  config.tolerance.atol));
    const auto started = std::chrono::steady_clock::now();

    std::vector<double> times(ts.steps);
    for (int64_t i = 0; i < ts.steps; i++) times[i] = ts.sample(i);
    if (!config.times.empty()) times = config.times;  // arbitrary output times

    // LogTolerance::from_linear (src/integrators/galpy/mod.rs:19-24)
    const double rtol_ln = std::log(config.tolerance.rtol);
    const double atol_ln = std::log(config.tolerance.atol);

    // Every stage's force sources are checked before any device work starts;
    // the origin tables of moving sources are built once their stage ran.
    std::vector<StageForce> forces(plan.stages.size());
    std::vector<std::vector<size_t>> moving(plan.stages.size());  // recipe indices
    for (size_t k = 0; k < plan.stages.size(); k++) {
        const Stage &stage = plan.stages[k];
        StageForce &f = forces[k];
        int n_static = 0;
        for (size_t i = 0; i < stage.recipes.size(); i++) {
            if (stage.recipe_is_background[i]) {
                f.model.statics[n_static++] = potential_of(stage.recipes[i]);
            } else if (config.attached_potentials) {
                if (!config.times.empty())
                    raise_not_implemented(fmt(
                        "stage %zu: potentials attached to particle groups need uniformly spaced "
                        "output times", k + 1));
                if (stage.container->t_end || stage.sources[i]->t_end)
                    raise_not_implemented(fmt(
                        "stage %zu: potentials attached to particle groups need the shared output grid "
                        "(no per-particle end times)", k + 1));
                moving[k].push_back(i);
            }
        }
        if (n_static == 0 && moving[k].empty())
            raise_not_implemented(fmt(
                "stage %zu has no force source: it requires no stationary background potential%s", k + 1,
                config.attached_potentials ? ""
                                           : " (potentials attached to particle groups act only with "
                                             "Config(attached_potentials=True))"));
        f.model.n_static = n_static;
        f.single = n_static == 1 && moving[k].empty();
        if (f.single) f.pot = f.model.statics[0];
    }
    std::vector<const Container *> stage_container;
    for (const Stage &st : plan.stages) stage_container.push_back(st.container);

    std::vector<py::object> results;
    // run(device=True): every buffer is a torch CUDA tensor on the current
    // device and stream, trajectories stay in HBM.
    py::object torch, dev, f64;
    uintptr_t stream = 0;
    if (device_out) {
        torch = py::module_::import("torch");
        if (!torch.attr("cuda").attr("is_available")().cast<bool>())
            throw DriftErrorCpp("GPU integration needs a CUDA device: torch.cuda is not available");
        dev = torch.attr("device")("cuda", torch.attr("cuda").attr("current_device")());
        f64 = torch.attr("float64");
        stream = torch.attr("cuda").attr("current_stream")(dev).attr("cuda_stream").cast<uintptr_t>();
    }
    auto to_device = [&](const double *data, py::ssize_t rows, py::ssize_t cols) {
        py::array_t<double> host(cols ? std::vector<py::ssize_t>{rows, cols} : std::vector<py::ssize_t>{rows});
        std::memcpy(host.mutable_data(), data, sizeof(double) * rows * (cols ? cols : 1));
        return torch.attr("from_numpy")(host).attr("to")(dev);
    };
    auto ptr_of = [](const py::object &t) { return t.attr("data_ptr")().cast<uintptr_t>(); };
    int64_t total_particles = 0;
    static bool backend_announced = false;
    int stage_no = 0;
    for (const Stage &stage : plan.stages) {
        stage_no++;
        const Container &c = *stage.container;
        const int64_t n = *c.num_particles;
        total_particles += n;
        DRIFT_LOG(LOG_GPU, LOG_DEBUG, fmt("stage %d: dispatching %lld particles to the GPU", stage_no, (long long)n));
        StageForce &force = forces[stage_no - 1];
        if (!moving[stage_no - 1].empty()) {
            // Origin tables of the moving sources, from their stages' trajectories.
            const int64_t nseg = ts.steps - 1;
            const double dt = (ts.end - ts.start) / (double)(ts.steps - 1);
            int64_t n_sources = 0;
            for (size_t i : moving[stage_no - 1]) n_sources += *stage.sources[i]->num_particles;
            if (device_out)
                force.origins_dev = torch.attr("empty")(py::make_tuple(nseg, n_sources, 18), "dtype"_a = f64,
                                                        "device"_a = dev);
            else
                force.origins.assign((size_t)nseg * n_sources * 18, 0.0);
            int64_t first = 0;
            int g = 0;
            for (size_t i : moving[stage_no - 1]) {
                const Container *src = stage.sources[i];
                size_t si = 0;
                while (si < stage_container.size() && stage_container[si] != src) si++;
                const int64_t ns = *src->num_particles;
                const drift_force_model src_model = forces[si].as_model();
                int rc;
                if (device_out) {
                    py::object part = torch.attr("empty")(py::make_tuple(nseg, ns, 18), "dtype"_a = f64,
                                                          "device"_a = dev);
                    const double *traj = reinterpret_cast<const double *>(ptr_of(results[si]));
                    double *dst = reinterpret_cast<double *>(ptr_of(part));
                    {
                        py::gil_scoped_release nogil;
                        rc = drift_origin_table(&src_model, ns, ts.steps, ts.start, dt, traj, dst,
                                                reinterpret_cast<void *>(stream));
                    }
                    if (rc == DRIFT_SUCCESS)
                        force.origins_dev.attr("__setitem__")(
                            py::make_tuple(py::slice(py::none(), py::none(), py::none()),
                                           py::slice(first, first + ns, 1)),
                            part);
                } else {
                    std::vector<double> part((size_t)nseg * ns * 18);
                    const double *traj = results[si].cast<py::array_t<double>>().data();
                    {
                        py::gil_scoped_release nogil;
                        rc = drift_origin_table_host(&src_model, ns, ts.steps, ts.start, dt, traj, part.data());
                    }
                    for (int64_t seg = 0; rc == DRIFT_SUCCESS && seg < nseg; seg++)
                        std::memcpy(force.origins.data() + ((size_t)seg * n_sources + first) * 18,
                                    part.data() + (size_t)seg * ns * 18, sizeof(double) * 18 * ns);
                }
                if (rc != DRIFT_SUCCESS)
                    throw IntegrationErrorCpp(fmt("origin table of stage %zu failed: %s (%s)", si + 1,
                                                  drift_result_string(rc), drift_last_error()));
                drift_source_group grp = source_group_of(stage.recipes[i]);
                grp.first = first;
                grp.count = ns;
                force.model.groups[g++] = grp;
                first += ns;
            }
            force.model.n_groups = g;
            force.model.n_sources = n_sources;
            force.model.n_segments = nseg;
            force.model.t0 = ts.start;
            force.model.dt = dt;
            force.model.origins = device_out ? reinterpret_cast<const double *>(ptr_of(force.origins_dev))
                                             : force.origins.data();
            DRIFT_LOG(LOG_GPU, LOG_DEBUG,
                      fmt("stage %d: force = %d stationary potential(s) + %d moving group(s) of %lld source particle(s)",
                          stage_no, force.model.n_static, g, (long long)n_sources));
        }

        drift_launch L;
        std::memset(&L, 0, sizeof(L));
        L.method = config.method == Method::DOPR54 ? DRIFT_DOPR54 : DRIFT_DOP853;
        L.precision = config.precision == Precision::EXACT ? DRIFT_PRECISION_EXACT : DRIFT_PRECISION_FMA;
        L.schedule = config.schedule == Schedule::PLAIN        ? DRIFT_SCHEDULE_PLAIN
                     : config.schedule == Schedule::PERSISTENT ? DRIFT_SCHEDULE_PERSISTENT
                                                               : DRIFT_SCHEDULE_ORDERED;
        L.block_size = config.block_size;
        if (force.single) {
            L.potential = force.pot;
        } else {
            L.potential.kind = DRIFT_POT_MODEL;
            L.force_model = &force.model;
        }
        L.n = n;
        L.y0 = c.state->data();
        L.nt = ts.steps;
        if (c.t_end) {
            L.ts = nullptr;
            L.t0 = ts.start;
            L.t_end = c.t_end->data();
        } else {
            L.ts = times.data();
        }
        L.rtol_ln = rtol_ln;
        L.atol_ln = atol_ln;
        L.dt_one = DRIFT_INITIAL_STEP_SENTINEL;
        L.max_steps = config.max_steps;
        L.timeout_s = config.timeout_s;
        L.arbitrary_times = config.arbitrary_times ? 1 : 0;

        py::array_t<uint8_t> status(n);
        py::array_t<int32_t> err(n);
        py::array_t<uint32_t> acc(n), rej(n);
        py::object out;
        // device mode: inputs, outputs and counters as CUDA tensors
        py::object y0_d, grid_d, st_d, err_d, acc_d, rej_d, ws_d;
        if (device_out) {
            y0_d = to_device(c.state->data(), n, STATE_DIM);
            grid_d = c.t_end ? to_device(c.t_end->data(), n, 0) : to_device(times.data(), ts.steps, 0);
            out = torch.attr("empty")(py::make_tuple(ts.steps, n, STATE_DIM), "dtype"_a = f64, "device"_a = dev);
            st_d = torch.attr("zeros")(n, "dtype"_a = torch.attr("uint8"), "device"_a = dev);
            err_d = torch.attr("zeros")(n, "dtype"_a = torch.attr("int32"), "device"_a = dev);
            acc_d = torch.attr("zeros")(n, "dtype"_a = torch.attr("int32"), "device"_a = dev);
            rej_d = torch.attr("zeros")(n, "dtype"_a = torch.attr("int32"), "device"_a = dev);
            L.y0 = reinterpret_cast<const double *>(ptr_of(y0_d));
            if (c.t_end)
                L.t_end = reinterpret_cast<const double *>(ptr_of(grid_d));
            else
                L.ts = reinterpret_cast<const double *>(ptr_of(grid_d));
            L.out = reinterpret_cast<double *>(ptr_of(out));
            L.status = reinterpret_cast<uint8_t *>(ptr_of(st_d));
            L.err_code = reinterpret_cast<int32_t *>(ptr_of(err_d));
            L.n_accepted = reinterpret_cast<uint32_t *>(ptr_of(acc_d));
            L.n_rejected = reinterpret_cast<uint32_t *>(ptr_of(rej_d));
            size_t ws_bytes = 0;
            drift_query_workspace(&L, &ws_bytes);
            if (ws_bytes) {
                ws_d = torch.attr("empty")(ws_bytes, "dtype"_a = torch.attr("uint8"), "device"_a = dev);
                L.workspace = reinterpret_cast<void *>(ptr_of(ws_d));
                L.workspace_bytes = ws_bytes;
            }
        } else {
            py::array_t<double> host_out({(py::ssize_t)ts.steps, (py::ssize_t)n, (py::ssize_t)STATE_DIM});
            L.out = host_out.mutable_data();
            L.status = status.mutable_data();
            L.err_code = err.mutable_data();
            L.n_accepted = acc.mutable_data();
            L.n_rejected = rej.mutable_data();
            out = host_out;
        }

        const char *kernel_label = config.method == Method::DOPR54 ? "GALPY DOPR54" : "GALPY DOP853";
        DRIFT_LOG(LOG_GPU, LOG_DEBUG,
                  fmt("launching %s kernel: %lld particles, block=%d, schedule=%s, %lld output times",
                      kernel_label, (long long)n, config.block_size ? config.block_size : 128,
                      config.schedule == Schedule::PLAIN        ? "plain"
                      : config.schedule == Schedule::PERSISTENT ? "persistent"
                                                                : "ordered",
                      (long long)ts.steps));
        if (!backend_announced) {
            DRIFT_LOG(LOG_BACKEND, LOG_DEBUG, "context initialized and kernel module loaded (sm_100a)");
            backend_announced = true;
        }
        const size_t in_bytes = n * STATE_DIM * sizeof(double) +
                                (c.t_end ? n : ts.steps) * sizeof(double);
        DRIFT_LOG(LOG_BACKEND, LOG_DEBUG, fmt("copying %zu bytes of host data to the device", in_bytes));

        const auto stage_started = std::chrono::steady_clock::now();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = device_out ? drift_integrate(&L, reinterpret_cast<void *>(stream)) : drift_integrate_host(&L);
        }
        if (device_out && rc == DRIFT_SUCCESS) {
            // the small per-particle counters come back (this also waits for the stage)
            auto fetch = [&](const py::object &t, auto &dst) {
                py::array a = t.attr("cpu")().attr("numpy")();
                std::memcpy(dst.mutable_data(), a.data(), a.nbytes());
            };
            fetch(st_d, status);
            fetch(err_d, err);
            fetch(acc_d, acc);
            fetch(rej_d, rej);
        }
        const double secs =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - stage_started).count();
        if (rc != DRIFT_SUCCESS) {
            std::string why = drift_last_error();
            if (rc == DRIFT_ERROR_NO_DEVICE) throw DriftErrorCpp("GPU integration needs a CUDA device: " + why);
            throw IntegrationErrorCpp(fmt("GPU %s integration failed: %s (%s)", name_of(config.method),
                                          drift_result_string(rc), why.c_str()));
        }
        const size_t out_bytes = (size_t)ts.steps * n * STATE_DIM * sizeof(double);
        if (device_out)
            DRIFT_LOG(LOG_BACKEND, LOG_DEBUG, fmt("kept %zu result bytes on the device", out_bytes));
        else
            DRIFT_LOG(LOG_BACKEND, LOG_DEBUG, fmt("copied %zu result bytes to the host", out_bytes));

        // galpy's DOPR54 error code first (the reference's CPU error), then
        // the build's own per-particle limits.
        const int32_t *e = err.data();
        const uint8_t *s = status.data();
        for (int64_t i = 0; i < n; i++)
            if (e[i] != 0)
                throw IntegrationErrorCpp(fmt("GPU %s integration failed with error code %d (particle %lld)",
                                              name_of(config.method), e[i], (long long)i));
        for (int64_t i = 0; i < n; i++)
            if (s[i] != DRIFT_PARTICLE_OK)
                throw IntegrationErrorCpp(fmt("GPU %s integration failed for particle %lld: %s",
                                              name_of(config.method), (long long)i, status_name(s[i])));

        DRIFT_LOG(LOG_GPU, LOG_DEBUG,
                  fmt("stage %d: %lld particles finished in %s", stage_no, (long long)n,
                      rust_duration(secs).c_str()));
        results.push_back(out);
        if (stats) stats->push_back(StageStats{acc, rej, status, secs, (uint64_t)in_bytes, (uint64_t)out_bytes});
    }
    const double elapsed =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
    DRIFT_LOG(LOG_GPU, LOG_INFO,
              fmt("GPU integration finished: %d stage(s), %lld particle trajectories in %s", stage_no,
                  (long long)total_particles, rust_duration(elapsed).c_str()));
    return results;
}

}  // namespace drift_host
