// The `cuda` vector-engine component: the plugin that a Bohrium stack loads with dlopen.
// Mirrors ve/cuda/main.cpp:42-168 of the reference (same messages, extmethod registration,
// memory-pointer semantics and repeat loop), with the B200 engine behind it.
#include <cstdint>
#include <iostream>
#include <sstream>
#include <string>
#include <bohrium/bh_component.hpp>
#include "engine.hpp"

using namespace std;
using namespace bohrium;
using namespace bohrium::component;

namespace {

class Impl : public ComponentVE {
public:
    cuda::EngineCUDA engine;

    explicit Impl(int stack_level) : ComponentVE(stack_level), engine(*this) {}
    ~Impl() override {
        if (engine.prof) cerr << engine.statistics();
    }

    void execute(BhIR *bhir) override {
        if (disabled) {
            child.execute(bhir);
            return;
        }
        engine.record_execute_begin();
        engine.execute(bhir);
        engine.record_execute_end();
    }

    void extmethod(const string &name, bh_opcode opcode) override {
        try {
            extmethods.insert(make_pair(opcode, extmethod::ExtmethodFace(config, name)));
        } catch (const extmethod::ExtmethodNotFound &) {
            if (!child.initiated()) throw;
            child.extmethod(name, opcode);
            child_extmethods.insert(opcode);
        }
    }

    string message(const string &msg) override {
        stringstream ss;
        if (msg == "statistic_enable_and_reset") {
            engine.resetStatistics();
            engine.prof = true;
        } else if (msg == "statistic") {
            ss << engine.statistics();
        } else if (msg == "GPU: disable") {
            engine.copyAllBasesToHost();
            disabled = true;
        } else if (msg == "GPU: enable") {
            disabled = false;
        } else if (msg == "CUDA: use current context") {
            // The engine always runs in the device's primary context, which every CUDA runtime
            // user in the process shares; nothing to switch.
        } else if (msg == "info") {
            ss << engine.info();
        } else if (msg == "CUDA: last execute ms") {
            ss.precision(9);
            ss << engine.last_execute_ms();
            return ss.str();
        } else if (msg == "CUDA: sync") {
            engine.synchronize_all();
        } else if (msg == "CUDA: timer start") {
            engine.timer_start();
        } else if (msg == "CUDA: timer stop") {
            ss.precision(9);
            ss << engine.timer_stop_ms();
            return ss.str();
        } else if (msg == "CUDA: launches") {
            ss << engine.stats().launches;
            return ss.str();
        } else if (msg.rfind("host_alloc ", 0) == 0) {
            ss << reinterpret_cast<uintptr_t>(engine.host_alloc(stoll(msg.substr(11))));
            return ss.str();
        } else if (msg.rfind("CUDA: batch ", 0) == 0) {
            engine.batch_mode = msg.substr(12);
        } else if (msg.rfind("CUDA: prof ", 0) == 0) {
            engine.prof = msg.substr(11) == "on";
        } else if (msg.rfind("CUDA: record ", 0) == 0) {
            engine.record = msg.substr(13) == "on";
        } else if (msg.rfind("CUDA: records dump ", 0) == 0) {
            ss << engine.dump_records(msg.substr(19));
            return ss.str();
        } else if (msg == "CUDA: records clear") {
            engine.clear_records();
        } else if (msg == "CUDA: records count") {
            ss << engine.record_count();
            return ss.str();
        } else if (msg.rfind("CUDA: costmodel load ", 0) == 0) {
            engine.load_costmodel(msg.substr(21));
        } else if (msg.rfind("CUDA: fuser ", 0) == 0) {
            engine.set_fusion("", msg.substr(12));
        } else if (msg.rfind("CUDA: pre_fuser ", 0) == 0) {
            engine.set_fusion(msg.substr(16), "");
        } else if (msg.rfind("CUDA: autotune ", 0) == 0) {
            engine.autotune = msg.substr(15) == "on";
        } else if (msg.rfind("CUDA: learned ", 0) == 0) {
            engine.learned_on = msg.substr(14) == "on";
        } else if (msg.rfind("CUDA: inject nvrtc ", 0) == 0) {
            engine.inject_nvrtc_failures = stoi(msg.substr(19));
        } else if (msg.rfind("CUDA: inject alloc ", 0) == 0) {
            engine.inject_alloc_failures = stoi(msg.substr(19));
        }
        return ss.str() + child.message(msg);
    }

    void *getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify) override {
        return engine.getMemoryPointer(base, copy2host, force_alloc, nullify);
    }

    void setMemoryPointer(bh_base *base, bool host_ptr, void *mem) override {
        engine.setMemoryPointer(base, host_ptr, mem);
    }

    void *getDeviceContext() override { return engine.stream(); }

    void setDeviceContext(void *) override {}

    string userKernel(const string &kernel, vector<bh_view> &operand_list, const string &compile_cmd,
                      const string &tag, const string &param) override {
        // The reference's ve/cuda throws for tag "cuda" (ve/cuda/main.cpp:111-121); this engine
        // compiles and runs the kernel on the device, as its OpenCL engine does for "opencl".
        if (tag == "cuda") return engine.userKernel(kernel, operand_list, param);
        for (const bh_view &op : operand_list) engine.copyToHost({op.base}, true);
        return child.userKernel(kernel, operand_list, compile_cmd, tag, param);
    }
};

} // namespace

extern "C" ComponentImpl *create(int stack_level) { return new Impl(stack_level); }
extern "C" void destroy(ComponentImpl *self) { delete self; }
