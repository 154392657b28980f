// tree.cpp -- container dependency graph (restates src/tree/mod.rs).
#include <atomic>

#include "model.h"

namespace drift_host {

const char *name_of(Engine e) { return e == Engine::CPU ? "CPU" : "GPU"; }
const char *name_of(Method m) { return m == Method::DOPR54 ? "DOPR54" : "DOP853"; }
const char *name_of(Implementation i)
{
    switch (i) {
    case Implementation::GALPY: return "GALPY";
    case Implementation::SCIPY: return "SCIPY";
    default: return "DRIFT";
    }
}

// Stable identities for containers (src/interface/container.rs:15-19).
uint64_t next_identity()
{
    static std::atomic<uint64_t> next{0};
    return next.fetch_add(1, std::memory_order_relaxed);
}

std::optional<std::vector<int>> AdjacencyMatrix::topological_order(
    const std::vector<bool> &present) const
{
    int indegree[N] = {0};
    for (int source = 0; source < N; source++)
        for (int dependent = 0; dependent < N; dependent++)
            if (present[source] && present[dependent] && get(source, dependent)) indegree[dependent]++;
    int count = 0;
    for (int i = 0; i < N; i++) count += present[i] ? 1 : 0;
    bool emitted[N] = {false};
    std::vector<int> order;
    order.reserve(count);
    while ((int)order.size() < count) {
        int next = -1;
        for (int node = 0; node < N; node++) {
            if (present[node] && !emitted[node] && indegree[node] == 0) {
                next = node;
                break;
            }
        }
        if (next < 0) return std::nullopt;
        emitted[next] = true;
        order.push_back(next);
        for (int dependent = 0; dependent < N; dependent++)
            if (present[dependent] && get(next, dependent)) indegree[dependent]--;
    }
    return order;
}

std::optional<IntegrationPlan> AdjacencyMatrix::build(
    const std::vector<const Container *> &by_label) const
{
    std::vector<bool> present(N, false);
    for (int i = 0; i < N && i < (int)by_label.size(); i++) present[i] = by_label[i] != nullptr;
    auto order = topological_order(present);
    if (!order) return std::nullopt;
    IntegrationPlan plan;
    for (int label : *order) {
        const Container *c = by_label[label];
        if (!c || !c->state) continue;  // backgrounds provide recipes, not stages
        Stage stage;
        stage.container = c;
        for (int source = 0; source < N && source < (int)by_label.size(); source++) {
            const Container *src = by_label[source];
            if (get(source, label) && src && src->recipe) {
                stage.recipes.push_back(*src->recipe);
                stage.recipe_is_background.push_back(!src->state);
                stage.sources.push_back(src);
            }
        }
        plan.stages.push_back(std::move(stage));
    }
    return plan;
}

}  // namespace drift_host
