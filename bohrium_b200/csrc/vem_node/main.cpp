// The `node` VEM: a pass-through component kept for stack parity with the reference
// (vem/node/main.cpp:29-95). With BH_MEM_WARN set it reports bases that were used but never
// freed when the component is destroyed.
#include <cstdlib>
#include <iostream>
#include <set>
#include <bohrium/bh_component.hpp>

using namespace std;
using namespace bohrium;
using namespace bohrium::component;

namespace {
class Impl : public ComponentImpl {
    set<const bh_base *> allocated;
    const bool mem_warn;

public:
    explicit Impl(int stack_level) : ComponentImpl(stack_level), mem_warn(getenv("BH_MEM_WARN") != nullptr) {}
    ~Impl() override {
        if (mem_warn && !allocated.empty())
            cerr << "[NODE-VEM] Warning: " << allocated.size() << " base arrays were not freed." << endl;
    }
    void execute(BhIR *bhir) override {
        if (mem_warn) {
            for (const bh_instruction &instr : bhir->instr_list) {
                if (instr.opcode == BH_FREE) {
                    allocated.erase(instr.operand[0].base);
                } else {
                    for (const bh_view &v : instr.getViews()) allocated.insert(v.base);
                }
            }
        }
        child.execute(bhir);
    }
};
} // namespace

extern "C" ComponentImpl *create(int stack_level) { return new Impl(stack_level); }
extern "C" void destroy(ComponentImpl *self) { delete self; }
