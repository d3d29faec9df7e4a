// The `bcexp` filter component (filter/bcexp/component_interface.cpp of the reference): rewrites
// each BhIR with bohrium::filter::expand (powk, sign, reduce1d) and passes it on. Options from
// the component's config section: powk (default true), sign (default false), reduce1d (the
// thread limit of the 1-D reduction split, default 0: off). Rewrites are made in
// place, so a re-executed BhIR is rewritten once; the temporaries that `sign` creates live as long
// as the component.
#include <bohrium/bh_component.hpp>
#include "../core/filters.hpp"

using namespace bohrium;
using namespace bohrium::component;

namespace {
class Impl : public ComponentImpl {
    filter::ExpandOptions opt;
    filter::BaseStore created;

public:
    explicit Impl(int stack_level) : ComponentImpl(stack_level) {
        opt.powk = config.defaultGet<bool>("powk", true);
        opt.sign = config.defaultGet<bool>("sign", false);
        opt.reduce1d = config.defaultGet<int64_t>("reduce1d", 0);
    }
    void execute(BhIR *bhir) override {
        filter::expand(*bhir, opt, created);
        child.execute(bhir);
    }
};
} // namespace

extern "C" ComponentImpl *create(int stack_level) { return new Impl(stack_level); }
extern "C" void destroy(ComponentImpl *self) { delete self; }
