// The `bccon` filter component (filter/bccon/component_interface.cpp of the reference): rewrites
// each BhIR with bohrium::filter::contract (stupidmath, collect, muladd) and passes it on.
// Options from the component's config section: stupidmath, collect, muladd (default true).
#include <bohrium/bh_component.hpp>
#include "../core/filters.hpp"

using namespace bohrium;
using namespace bohrium::component;

namespace {
class Impl : public ComponentImpl {
    filter::ContractOptions opt;

public:
    explicit Impl(int stack_level) : ComponentImpl(stack_level) {
        opt.stupidmath = config.defaultGet<bool>("stupidmath", true);
        opt.collect = config.defaultGet<bool>("collect", true);
        opt.muladd = config.defaultGet<bool>("muladd", true);
    }
    void execute(BhIR *bhir) override {
        filter::contract(*bhir, opt);
        child.execute(bhir);
    }
};
} // namespace

extern "C" ComponentImpl *create(int stack_level) { return new Impl(stack_level); }
extern "C" void destroy(ComponentImpl *self) { delete self; }
