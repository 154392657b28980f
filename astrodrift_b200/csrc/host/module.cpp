// module.cpp -- pybind11 module `astrodrift_b200._drift`: the drift Python
// surface (Config / Potential / Container / test_particles / particles /
// background / DriftError / IntegrationError) over the C++ host layer.
//
// Restates src/interface/mod.rs (PyOutputGrid :29-132, PyTolerance :137-171,
// PyConfig :178-469), src/interface/container.rs, src/interface/recipe.rs,
// src/interface/selector.rs and src/interface/error.rs, keeping their names,
// argument meaning, validation messages and exception types.  Additive
// extensions: Config(precision=, schedule=, block_size=, max_steps=,
// timeout=, attached_potentials=, arbitrary_times=), run(stats=True, device=True), test_particles/particles(t_end=) and
// Potential.bovy(keyword parameters).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <cstdio>
#include <limits>
#include <optional>
#include <string>
#include <vector>

#include "dispatch.h"
#include "drift_b200.h"
#include "model.h"

namespace py = pybind11;
using namespace drift_host;

namespace {

std::string py_float(double v)
{
    if (std::isnan(v)) return "float('nan')";
    if (std::isinf(v)) return v > 0 ? "float('inf')" : "float('-inf')";
    return py::repr(py::float_(v)).cast<std::string>();
}

// selector.rs:4-22: selectors must be exact members of drift's StrEnums.
std::string extract_selector(const py::handle &obj, const char *name)
{
    py::object cls = py::module_::import("astrodrift_b200.selectors").attr(name);
    if (!obj.get_type().is(cls))
        throw py::type_error(std::string("expected a drift.") + name + " member");
    try {
        return obj.attr("value").cast<std::string>();
    } catch (const py::cast_error &) {
        throw py::value_error(std::string("invalid ") + name + " value");
    }
}

constexpr double GRID_ULP_TOLERANCE = 8.0;

OutputGrid grid_new(double start, double end, int64_t steps)
{
    if (steps < 2 || steps > MAX_OUTPUT_TIMES)
        throw py::value_error("ts must contain between 2 and " + std::to_string(MAX_OUTPUT_TIMES) +
                              " output times");
    if (!std::isfinite(start) || !std::isfinite(end)) throw py::value_error("ts endpoints must be finite");
    double span = end - start;
    if (span == 0.0 || !std::isfinite(span))
        throw py::value_error("ts must span a non-zero finite interval");
    return OutputGrid{start, end, steps};
}

OutputGrid grid_from_times(const double *t, int64_t len, bool uniform = true)
{
    if (len < 2 || len > MAX_OUTPUT_TIMES)
        throw py::value_error("ts must contain between 2 and " + std::to_string(MAX_OUTPUT_TIMES) +
                              " output times");
    for (int64_t i = 0; i < len; i++)
        if (!std::isfinite(t[i])) throw py::value_error("all ts values must be finite");
    OutputGrid g = grid_new(t[0], t[len - 1], len);
    bool increasing = g.end > g.start;
    for (int64_t i = 0; i + 1 < len; i++)
        if (increasing ? t[i + 1] <= t[i] : t[i + 1] >= t[i])
            throw py::value_error("ts values must be strictly increasing or strictly decreasing");
    if (!uniform) return g;
    double step = (g.end - g.start) / (double)(g.steps - 1);
    for (int64_t i = 0; i < len; i++) {
        double expected = g.sample(i);
        double scale = std::max({std::fabs(t[i]), std::fabs(expected), std::fabs(step),
                                 std::numeric_limits<double>::min()});
        double tol = GRID_ULP_TOLERANCE * std::numeric_limits<double>::epsilon() * scale;
        if (std::fabs(t[i] - expected) > tol)
            throw py::value_error(
                "ts values must be uniformly spaced; arbitrary output times are not yet supported");
    }
    return g;
}

// PyOutputGrid::extract (src/interface/mod.rs:31-65)
// With `times` (Config(arbitrary_times=True)), explicit time lists need only
// be finite and strictly monotone, and are kept as given.
OutputGrid extract_grid(const py::handle &obj, std::vector<double> *times = nullptr)
{
    if (py::isinstance<py::tuple>(obj)) {
        py::tuple tup = obj.cast<py::tuple>();
        if (tup.size() != 3)
            throw py::value_error("time-grid tuple must have 3 elements: (start, end, steps)");
        return grid_new(tup[0].cast<double>(), tup[1].cast<double>(), tup[2].cast<int64_t>());
    }
    if (py::isinstance<py::array>(obj)) {
        py::array arr = obj.cast<py::array>();
        if (arr.ndim() == 1 && arr.dtype().is(py::dtype::of<double>())) {
            if (!(arr.flags() & py::array::c_style))
                throw py::value_error("NumPy time arrays must be contiguous");
            const double *t = static_cast<const double *>(arr.data());
            OutputGrid g = grid_from_times(t, arr.shape(0), times == nullptr);
            if (times) times->assign(t, t + arr.shape(0));
            return g;
        }
    }
    try {
        std::vector<double> seq = obj.cast<std::vector<double>>();
        OutputGrid g = grid_from_times(seq.data(), (int64_t)seq.size(), times == nullptr);
        if (times) *times = seq;
        return g;
    } catch (const py::cast_error &) {
    }
    throw py::value_error("Expected (start, end, steps) tuple or 1D numpy.linspace array");
}

Tolerance tolerance_new(double rtol, double atol)
{
    if (!std::isfinite(rtol) || !std::isfinite(atol) || rtol <= 0.0 || atol <= 0.0)
        throw py::value_error("rtol and atol must be finite and greater than zero");
    return Tolerance{rtol, atol};
}

// PyTolerance::extract (src/interface/mod.rs:139-159)
Tolerance extract_tolerance(const py::handle &obj)
{
    if (py::isinstance<py::tuple>(obj)) {
        py::tuple tup = obj.cast<py::tuple>();
        if (tup.size() == 2) return tolerance_new(tup[0].cast<double>(), tup[1].cast<double>());
    }
    try {
        double v = obj.cast<double>();
        return tolerance_new(v, v);
    } catch (const py::cast_error &) {
    }
    throw py::value_error("Expected (rtol, atol) tuple or single float tolerance value");
}

// validate_configuration (src/integrators/mod.rs:23-36).  This package
// integrates on the GPU only; the reference's CPU engine is its own
// line-by-line host port, which this package keeps as a test oracle rather
// than as a product path.
void validate_configuration(const Config &c)
{
    bool ok = c.engine == Engine::GPU && c.implementation == Implementation::GALPY;
    if (!ok)
        raise_not_implemented(std::string(name_of(c.engine)) + " + " + name_of(c.implementation) + " " +
                              name_of(c.method) + " is not implemented");
}

std::string recipe_repr(const Recipe &r)
{
    switch (r.name) {
    case PotentialName::Kepler:
    case PotentialName::CustomKepler:
        return "Potential.kepler(amp=" + py_float(r.amp) + ")";
    case PotentialName::Plummer:
    case PotentialName::CustomPlummer:
        return "Potential.plummer(amp=" + py_float(r.amp) + ", radius=" + py_float(r.radius) + ")";
    default:
        return "Potential.bovy()";
    }
}

// validate_istate (src/interface/container.rs:55-93)
std::shared_ptr<const std::vector<double>> validate_istate(const py::array &istate, int64_t *count)
{
    py::array_t<double, py::array::c_style | py::array::forcecast> a(istate);
    std::vector<py::ssize_t> shape(a.shape(), a.shape() + a.ndim());
    int64_t particles = 0;
    bool well_formed = false;
    if (shape.size() == 1) {
        particles = shape[0] / STATE_DIM;
        well_formed = shape[0] % STATE_DIM == 0;
    } else if (shape.size() == 2) {
        particles = shape[0];
        well_formed = shape[1] == STATE_DIM;
    }
    if (!well_formed) {
        std::string s = "[";
        for (size_t i = 0; i < shape.size(); i++) s += (i ? ", " : "") + std::to_string(shape[i]);
        s += "]";
        throw py::value_error(
            "istate must have shape (N, 6) with columns [x, y, z, vx, vy, vz] (or a flat array of length 6N); got shape " + s);
    }
    if (particles == 0) throw py::value_error("istate must contain at least one particle");
    if (particles > MAX_PARTICLES)
        throw py::value_error("istate has " + std::to_string(particles) +
                              " particles but the current engine supports at most " +
                              std::to_string(MAX_PARTICLES) + "; split the group into multiple containers");
    const double *d = a.data();
    const int64_t len = particles * STATE_DIM;
    for (int64_t i = 0; i < len; i++)
        if (!std::isfinite(d[i])) throw py::value_error("istate positions and velocities must be finite");
    *count = particles;
    return std::make_shared<const std::vector<double>>(d, d + len);
}

std::shared_ptr<const std::vector<double>> validate_t_end(const py::object &t_end, int64_t n)
{
    if (t_end.is_none()) return nullptr;
    py::array_t<double, py::array::c_style | py::array::forcecast> a(t_end);
    if (a.ndim() != 1 || a.shape(0) != n)
        throw py::value_error("t_end must be a 1-D array with one end time per particle");
    const double *d = a.data();
    for (int64_t i = 0; i < n; i++)
        if (!std::isfinite(d[i])) throw py::value_error("t_end values must be finite");
    return std::make_shared<const std::vector<double>>(d, d + n);
}

struct ConfigObject {
    Config inner;
    std::vector<std::pair<uint64_t, uint64_t>> dependencies;  // (source, dependent)
    std::vector<Container> containers;

    static void register_container(std::vector<Container> &cs, const Container &c)
    {
        for (const auto &x : cs)
            if (x.identity == c.identity) return;
        cs.push_back(c);
    }

    bool dependency_path_exists(uint64_t start, uint64_t target) const
    {
        std::vector<uint64_t> pending{start}, visited;
        while (!pending.empty()) {
            uint64_t cur = pending.back();
            pending.pop_back();
            if (cur == target) return true;
            if (std::find(visited.begin(), visited.end(), cur) != visited.end()) continue;
            visited.push_back(cur);
            for (auto &e : dependencies)
                if (e.first == cur) pending.push_back(e.second);
        }
        return false;
    }

    void add_dependencies(uint64_t node, const std::vector<uint64_t> &requires_)
    {
        if (requires_.empty()) throw py::value_error("add() requires at least one dependency");
        for (uint64_t d : requires_)
            if (dependency_path_exists(node, d))
                throw py::value_error("adding these dependencies would create a cycle");
        for (uint64_t d : requires_) {
            std::pair<uint64_t, uint64_t> edge{d, node};
            if (std::find(dependencies.begin(), dependencies.end(), edge) == dependencies.end())
                dependencies.push_back(edge);
        }
    }

    void add(const Container &node, const py::args &requires_)
    {
        std::vector<uint64_t> ids;
        std::vector<Container> deps;
        for (const auto &obj : requires_) {
            const Container &c = obj.cast<const Container &>();
            if (std::find(ids.begin(), ids.end(), c.identity) == ids.end()) {
                ids.push_back(c.identity);
                deps.push_back(c);
            }
        }
        std::vector<Container> cs = containers;
        register_container(cs, node);
        for (const auto &d : deps) register_container(cs, d);
        if ((int64_t)cs.size() > MAX_MODEL_COMPONENTS)
            throw py::value_error("add() would register " + std::to_string(cs.size()) +
                                  " containers but a model supports at most " +
                                  std::to_string(MAX_MODEL_COMPONENTS));
        add_dependencies(node.identity, ids);
        containers = cs;
    }

    void validate_registered_model() const
    {
        for (const auto &c : containers) {
            if (!c.state) continue;
            bool has_incoming = false;
            for (auto &e : dependencies)
                if (e.second == c.identity) has_incoming = true;
            if (!has_incoming)
                throw py::value_error(
                    "each particle container must be registered with add(node, *requires) before integration");
        }
    }

    IntegrationPlan build_tree() const
    {
        std::vector<const Container *> by_label(MAX_MODEL_COMPONENTS, nullptr);
        std::vector<uint64_t> ids;
        for (size_t label = 0; label < containers.size(); label++) {
            if (std::find(ids.begin(), ids.end(), containers[label].identity) != ids.end())
                throw py::value_error("run() received the same container more than once");
            ids.push_back(containers[label].identity);
            by_label[label] = &containers[label];
        }
        AdjacencyMatrix adj;
        for (auto &e : dependencies) {
            auto node = std::find(ids.begin(), ids.end(), e.second);
            auto dep = std::find(ids.begin(), ids.end(), e.first);
            if (node == ids.end()) throw DriftErrorCpp("registered node is missing");
            if (dep == ids.end()) throw DriftErrorCpp("registered dependency is missing");
            adj.set((int)(dep - ids.begin()), (int)(node - ids.begin()), true);
        }
        auto plan = adj.build(by_label);
        if (!plan) throw py::value_error("container dependencies must form an acyclic graph");
        return *plan;
    }

    py::object run(bool want_stats, bool device)
    {
        validate_registered_model();
        IntegrationPlan plan = build_tree();
        validate_configuration(inner);
        std::vector<StageStats> stats;
        std::vector<py::object> results;
        if (!plan.stages.empty()) results = gpu_dispatch(inner, plan, want_stats ? &stats : nullptr, device);
        py::list items;
        py::list stat_items;
        for (const auto &c : containers) {
            py::object item = py::none();
            py::object st = py::none();
            for (size_t s = 0; s < plan.stages.size(); s++) {
                if (plan.stages[s].container->identity == c.identity) {
                    item = results[s];
                    if (want_stats) {
                        py::dict d;
                        d["accepted"] = stats[s].accepted;
                        d["rejected"] = stats[s].rejected;
                        d["status"] = stats[s].status;
                        d["seconds"] = stats[s].seconds;
                        d["bytes_in"] = stats[s].bytes_in;
                        d["bytes_written"] = stats[s].bytes_written;
                        st = d;
                    }
                }
            }
            if (item.is_none() && c.state)
                throw DriftErrorCpp("integration returned no output for a particle container");
            items.append(item);
            stat_items.append(st);
        }
        if (want_stats) return py::make_tuple(items, stat_items);
        return items;
    }

    std::string info() const
    {
        char tol[96];
        std::snprintf(tol, sizeof(tol), "tolerance=(rtol=%.6e, atol=%.6e)", inner.tolerance.rtol,
                      inner.tolerance.atol);
        auto num = [](double v) {
            py::object f = py::float_(v);
            if (std::isfinite(v) && v == std::floor(v) && std::fabs(v) < 1e16)
                return std::to_string((long long)v);
            return py::repr(f).cast<std::string>();
        };
        return std::string("Config(engine=") + name_of(inner.engine) + ", method=" + name_of(inner.method) +
               ", implementation=" + name_of(inner.implementation) + ", times=(" + num(inner.output.start) +
               ", " + num(inner.output.end) + ", " + std::to_string(inner.output.steps) + "), " + tol +
               ", containers=" + std::to_string(containers.size()) +
               ", dependencies=" + std::to_string(dependencies.size()) + ")";
    }
};

Container make_particles(const py::array &istate, std::optional<Recipe> recipe, const py::object &t_end)
{
    Container c;
    int64_t n = 0;
    c.state = validate_istate(istate, &n);
    c.num_particles = n;
    c.recipe = recipe;
    c.t_end = validate_t_end(t_end, n);
    c.identity = next_identity();
    return c;
}

}  // namespace

PYBIND11_MODULE(_drift, m)
{
    m.doc() = "B200-native drift integration path: configuration, containers and GPU dispatch.";
    m.attr("_cuda_compiler") = "nvcc-sm_100a";
    m.attr("MAX_MODEL_COMPONENTS") = MAX_MODEL_COMPONENTS;
    m.attr("MAX_PARTICLES") = MAX_PARTICLES;
    m.attr("MAX_OUTPUT_TIMES") = MAX_OUTPUT_TIMES;

    static py::exception<DriftErrorCpp> drift_error(m, "DriftError", PyExc_RuntimeError);
    static py::exception<IntegrationErrorCpp> integration_error(m, "IntegrationError", drift_error.ptr());
    py::register_exception_translator([](std::exception_ptr p) {
        try {
            if (p) std::rethrow_exception(p);
        } catch (const IntegrationErrorCpp &e) {
            py::set_error(integration_error, e.what());
        } catch (const DriftErrorCpp &e) {
            py::set_error(drift_error, e.what());
        }
    });

    py::class_<Recipe>(m, "Potential", "A gravitational potential definition.")
        .def_static(
            "kepler",
            [](double amp) {
                Recipe r;
                r.name = PotentialName::Kepler;
                r.amp = amp;
                return r;
            },
            py::arg("amp"), "Point-mass potential with total mass ``amp`` (G = 1).")
        .def_static(
            "plummer",
            [](double amp, double radius) {
                Recipe r;
                r.name = PotentialName::Plummer;
                r.amp = amp;
                r.radius = radius;
                return r;
            },
            py::arg("amp"), py::arg("radius"), "Plummer sphere with mass ``amp`` and scale radius ``radius``.")
        .def_static(
            "bovy",
            [](double disk_amp, double disk_a, double disk_b, double halo_amp, double halo_a,
               double bulge_alpha, double bulge_rc, double bulge_force) {
                Recipe r;
                r.name = PotentialName::Bovy;
                r.mn_amp = disk_amp;
                r.mn_a = disk_a;
                r.mn_b = disk_b;
                r.nfw_amp = halo_amp;
                r.nfw_a = halo_a;
                r.bulge_alpha = bulge_alpha;
                r.bulge_rc = bulge_rc;
                r.bulge_force = bulge_force;
                return r;
            },
            py::kw_only(), py::arg("disk_amp") = 0.7574802019, py::arg("disk_a") = 3.0 / 8.0,
            py::arg("disk_b") = 0.28 / 8.0, py::arg("halo_amp") = 4.852230533528,
            py::arg("halo_a") = 16.0 / 8.0, py::arg("bulge_alpha") = 1.8,
            py::arg("bulge_rc") = 1.9 / 8.0, py::arg("bulge_force") = 0.05,
            "The built-in composite: power-law bulge with cutoff + Miyamoto-Nagai disk + NFW halo.")
        .def("__repr__", &recipe_repr)
        .def_property_readonly("parameters", [](const Recipe &r) {
            py::dict d;
            d["amp"] = r.amp;
            d["radius"] = r.radius;
            d["disk_amp"] = r.mn_amp;
            d["disk_a"] = r.mn_a;
            d["disk_b"] = r.mn_b;
            d["halo_amp"] = r.nfw_amp;
            d["halo_a"] = r.nfw_a;
            d["bulge_alpha"] = r.bulge_alpha;
            d["bulge_rc"] = r.bulge_rc;
            d["bulge_force"] = r.bulge_force;
            d["kind"] = (int)r.name;
            return d;
        });

    py::class_<Container>(m, "Container", "A state-bearing particle group or stationary background potential.")
        .def_property_readonly("num_particles",
                               [](const Container &c) -> py::object {
                                   if (c.num_particles) return py::int_(*c.num_particles);
                                   return py::none();
                               })
        .def("__repr__", [](const Container &c) {
            if (c.num_particles && c.recipe)
                return "Container(kind='particles', num_particles=" + std::to_string(*c.num_particles) +
                       ", potential=" + recipe_repr(*c.recipe) + ")";
            if (c.num_particles)
                return "Container(kind='test_particles', num_particles=" + std::to_string(*c.num_particles) + ")";
            if (c.recipe) return "Container(kind='background', potential=" + recipe_repr(*c.recipe) + ")";
            return std::string("Container(kind='background', potential=None)");
        });

    m.def(
        "test_particles",
        [](const py::array &istate, const py::object &t_end) {
            return make_particles(istate, std::nullopt, t_end);
        },
        py::arg("istate"), py::kw_only(), py::arg("t_end") = py::none(),
        "A state-bearing particle group without an attached potential.");
    m.def(
        "particles",
        [](const Recipe &potential, const py::array &istate, const py::object &t_end) {
            Recipe r = potential;
            if (r.name == PotentialName::Kepler)
                r.name = PotentialName::CustomKepler;
            else if (r.name == PotentialName::Plummer)
                r.name = PotentialName::CustomPlummer;
            else
                raise_not_implemented("only Kepler and Plummer potentials can currently be attached to particles");
            return make_particles(istate, r, t_end);
        },
        py::arg("potential"), py::arg("istate"), py::kw_only(), py::arg("t_end") = py::none(),
        "A state-bearing particle group with an attached potential.");
    m.def(
        "background",
        [](const Recipe &potential) {
            Container c;
            c.recipe = potential;
            c.identity = next_identity();
            return c;
        },
        py::arg("potential"), "A stationary background potential for use as a force source.");

    py::class_<ConfigObject>(m, "Config", "Configuration and registered container graph for an integration.")
        .def(py::init([](py::object engine, py::object method, py::object implementation, py::object ts,
                         py::object tolerance, py::object precision, py::object schedule, int block_size,
                         int64_t max_steps, double timeout, bool attached_potentials,
                         bool arbitrary_times) {
                 ConfigObject c;
                 if (!engine.is_none()) c.inner.engine = extract_selector(engine, "Engine") == "CPU" ? Engine::CPU : Engine::GPU;
                 if (!method.is_none()) {
                     std::string v = extract_selector(method, "Method");
                     if (v == "DOPR54")
                         c.inner.method = Method::DOPR54;
                     else if (v == "DOP853")
                         c.inner.method = Method::DOP853;
                     else
                         throw py::value_error("invalid Method value");
                 }
                 if (!implementation.is_none()) {
                     std::string v = extract_selector(implementation, "Implementation");
                     if (v == "GALPY")
                         c.inner.implementation = Implementation::GALPY;
                     else if (v == "SCIPY")
                         c.inner.implementation = Implementation::SCIPY;
                     else if (v == "DRIFT")
                         c.inner.implementation = Implementation::DRIFT;
                     else
                         throw py::value_error("invalid Implementation value");
                 }
                 c.inner.arbitrary_times = arbitrary_times;
                 if (!ts.is_none())
                     c.inner.output = extract_grid(ts, arbitrary_times ? &c.inner.times : nullptr);
                 if (!tolerance.is_none()) c.inner.tolerance = extract_tolerance(tolerance);
                 if (!precision.is_none()) {
                     std::string v = precision.cast<std::string>();
                     if (v == "exact")
                         c.inner.precision = Precision::EXACT;
                     else if (v == "fma")
                         c.inner.precision = Precision::FMA;
                     else
                         throw py::value_error("precision must be 'exact' or 'fma'");
                 }
                 if (!schedule.is_none()) {
                     std::string v = schedule.cast<std::string>();
                     if (v == "plain")
                         c.inner.schedule = Schedule::PLAIN;
                     else if (v == "persistent")
                         c.inner.schedule = Schedule::PERSISTENT;
                     else if (v == "ordered")
                         c.inner.schedule = Schedule::ORDERED;
                     else
                         throw py::value_error("schedule must be 'plain', 'persistent' or 'ordered'");
                 }
                 if (block_size != 0 && (block_size < 32 || block_size > 128 || block_size % 32))
                     throw py::value_error("block_size must be a multiple of 32 in [32, 128]");
                 c.inner.block_size = block_size;
                 c.inner.max_steps = max_steps;
                 c.inner.timeout_s = timeout;
                 c.inner.attached_potentials = attached_potentials;
                 validate_configuration(c.inner);
                 return c;
             }),
             py::arg("engine") = py::none(), py::arg("method") = py::none(),
             py::arg("implementation") = py::none(), py::arg("ts") = py::none(),
             py::arg("tolerance") = py::none(), py::kw_only(), py::arg("precision") = py::none(),
             py::arg("schedule") = py::none(), py::arg("block_size") = 0, py::arg("max_steps") = 0,
             py::arg("timeout") = 0.0, py::arg("attached_potentials") = false,
             py::arg("arbitrary_times") = false)
        .def("run", &ConfigObject::run, py::kw_only(), py::arg("stats") = false, py::arg("device") = false,
             "Integrate the registered model; results follow first-registration order.  "
             "device=True returns torch CUDA tensors that the kernels wrote in place.")
        .def("add", &ConfigObject::add, py::arg("node"),
             "Register force-source edges from ``requires`` to ``node``.")
        .def(
            "dependency",
            [](ConfigObject &self, const Container &node, const py::args &requires_) {
                if (PyErr_WarnEx(PyExc_DeprecationWarning,
                                 "Config.dependency() is deprecated; use Config.add(node, *requires)", 1) < 0)
                    throw py::error_already_set();
                self.add(node, requires_);
            },
            py::arg("node"), "Deprecated alias for :meth:`add`.")
        .def("info", &ConfigObject::info)
        .def("__repr__", &ConfigObject::info);

    m.def("abi_version", &drift_abi_version);
}
