// model.h -- configuration, potentials ("recipes"), containers and the
// container dependency graph of the drift integration path.
//
// Restates the reference's host data model in C++:
//   Config / OutputGrid / Tolerance         shared/src/config.rs:5-125
//   Recipe and PotentialName                 shared/src/model.rs:482-600
//   Container                                src/interface/container.rs:21-53
//   AdjacencyMatrix / IntegrationPlan        src/tree/mod.rs:6-117
// with the per-container particle and output-time caps lifted (the reference
// caps particles at 1000 and output times at 1024, shared/src/lib.rs:25-27).
#pragma once

#include <cstdint>
#include <memory>
#include <optional>
#include <string>
#include <vector>

namespace drift_host {

enum class Engine { CPU, GPU };
enum class Method { DOPR54, DOP853 };
enum class Implementation { GALPY, SCIPY, DRIFT };
enum class Precision { EXACT, FMA };
enum class Schedule { PLAIN, PERSISTENT, ORDERED };

const char *name_of(Engine e);
const char *name_of(Method m);
const char *name_of(Implementation i);

// shared/src/lib.rs:21-41, with the particle / output-time caps raised to what
// one GPU's memory can hold.
constexpr int64_t MAX_MODEL_COMPONENTS = 11;
constexpr int64_t MAX_PARTICLES = int64_t(1) << 30;
constexpr int64_t MAX_OUTPUT_TIMES = int64_t(1) << 24;
constexpr double MIN_RTOL = 1e-12;
constexpr double MIN_ATOL = 1e-12;
constexpr int STATE_DIM = 6;

// Inclusive affine output grid (shared/src/config.rs:55-67).
struct OutputGrid {
    double start = 0.0;
    double end = 6.283185307179586;  // 2 pi
    int64_t steps = 100;
    double sample(int64_t index) const
    {
        if (index == steps - 1) return end;
        return start + (end - start) * (double)index / (double)(steps - 1);
    }
};

struct Tolerance {
    double rtol = MIN_RTOL;
    double atol = MIN_ATOL;
};

struct Config {
    // The B200 build integrates on the GPU; see interface validation.
    Engine engine = Engine::GPU;
    Method method = Method::DOPR54;
    Implementation implementation = Implementation::GALPY;
    OutputGrid output;
    Tolerance tolerance;
    Precision precision = Precision::EXACT;
    Schedule schedule = Schedule::ORDERED;
    int block_size = 0;
    int64_t max_steps = 0;
    double timeout_s = 0.0;
    // Potentials attached to required particle groups act as moving force
    // sources.  Off by default: the reference does not build them yet
    // (shared/src/model.rs:193-199) and its tests expect them to exert no force.
    bool attached_potentials = false;
    // Output times kept as given (Config(arbitrary_times=True) with a time
    // list): need not be uniform.  Empty: the affine grid `output`.
    bool arbitrary_times = false;
    std::vector<double> times;
};

enum class PotentialName { Kepler, Plummer, Bovy, CustomKepler, CustomPlummer };

// A potential definition (shared/src/model.rs:482-600).  Bovy carries its
// disk and halo parameters so they can be varied.
struct Recipe {
    PotentialName name = PotentialName::Kepler;
    double amp = 1.0;
    double radius = 0.0;
    double mn_amp = 0.7574802019, mn_a = 3.0 / 8.0, mn_b = 0.28 / 8.0;
    double nfw_amp = 4.852230533528, nfw_a = 16.0 / 8.0;
    double bulge_alpha = 1.8, bulge_rc = 1.9 / 8.0, bulge_force = 0.05;
};

// A state-bearing particle group or a stationary background potential.
struct Container {
    std::optional<int64_t> num_particles;
    std::optional<Recipe> recipe;
    std::shared_ptr<const std::vector<double>> state;       // (N, 6) initial states
    std::shared_ptr<const std::vector<double>> t_end;       // optional per-particle end times
    uint64_t identity = 0;
};

uint64_t next_identity();

// One integration stage: a state-bearing container and the recipes of the
// containers it requires (src/tree/mod.rs:89-110).
struct Stage {
    const Container *container = nullptr;
    std::vector<Recipe> recipes;
    std::vector<bool> recipe_is_background;
    std::vector<const Container *> sources;  // the container each recipe comes from
};

struct IntegrationPlan {
    std::vector<Stage> stages;  // topological (dependency) order
};

// Packed row-major 11 x 11 bitset where (source, dependent) marks a force
// input (src/tree/mod.rs:14-42).
struct AdjacencyMatrix {
    unsigned __int128 bits = 0;
    static constexpr int N = (int)MAX_MODEL_COMPONENTS;
    bool get(int r, int c) const { return ((bits >> (r * N + c)) & 1) != 0; }
    void set(int r, int c, bool v)
    {
        unsigned __int128 bit = (unsigned __int128)1 << (r * N + c);
        if (v)
            bits |= bit;
        else
            bits &= ~bit;
    }
    // Stable Kahn topological sort choosing the lowest label on ties
    // (src/tree/mod.rs:44-73).  Empty optional: the graph has a cycle.
    std::optional<std::vector<int>> topological_order(const std::vector<bool> &present) const;
    // Stages in dependency order (src/tree/mod.rs:75-117).
    std::optional<IntegrationPlan> build(const std::vector<const Container *> &by_label) const;
};

}  // namespace drift_host
