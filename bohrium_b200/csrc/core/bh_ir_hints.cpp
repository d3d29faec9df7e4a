// The process-wide side table of BhIR execution hints (include/bohrium/bh_ir.hpp). It has no
// counterpart in the reference, whose BhIR carries no hints.
#include <mutex>
#include <unordered_map>
#include <bohrium/bh_ir.hpp>

namespace {
std::mutex g_mutex;
std::unordered_map<const BhIR *, BhIRHints> &table() {
    static std::unordered_map<const BhIR *, BhIRHints> t;
    return t;
}
} // namespace

void bh_ir_hints_set(const BhIR *ir, const BhIRHints &hints) {
    std::lock_guard<std::mutex> lock(g_mutex);
    table()[ir] = hints;
}

BhIRHints bh_ir_hints_get(const BhIR *ir) {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = table().find(ir);
    return it == table().end() ? BhIRHints() : it->second;
}

void bh_ir_hints_clear(const BhIR *ir) {
    std::lock_guard<std::mutex> lock(g_mutex);
    table().erase(ir);
}
