// The Bohrium component plugin interface.
//
// Same classes, members and virtual methods (in the same order) as
// include/bohrium/bh_component.hpp:51-264 of the reference: a component is a shared library that
// exports
//     extern "C" ComponentImpl* create(int stack_level);
//     extern "C" void destroy(ComponentImpl* self);
// and ComponentFace dlopen()s it (core/bh_component.cpp:30-61). Each ComponentImpl reads its
// config section, then creates its child (the next entry of the stack list).
#pragma once

#include <map>
#include <set>
#include <string>
#include <vector>
#include <bohrium/bh_config_parser.hpp>
#include <bohrium/bh_ir.hpp>
#include <bohrium/bh_opcode.h>
#include <bohrium/bh_extmethod.hpp>

namespace bohrium {
namespace component {

class ComponentImpl;

class ComponentFace {
    void *_lib_handle = nullptr;
    ComponentImpl *_implementation = nullptr;
    ComponentImpl *(*_create)(int) = nullptr;
    void (*_destroy)(ComponentImpl *component) = nullptr;

public:
    ComponentFace(const std::string &lib_path, int stack_level);
    ComponentFace() = default;
    ComponentFace(const ComponentFace &other) = delete;
    ComponentFace(ComponentFace &&other) = delete;
    ~ComponentFace();
    ComponentFace &operator=(ComponentFace &&other) noexcept {
        _lib_handle = other._lib_handle;
        _implementation = other._implementation;
        _create = other._create;
        _destroy = other._destroy;
        other._lib_handle = nullptr;
        other._implementation = nullptr;
        other._create = nullptr;
        other._destroy = nullptr;
        return *this;
    }

    virtual bool initiated() const;
    virtual void execute(BhIR *bhir);
    virtual void extmethod(const std::string &name, bh_opcode opcode);
    virtual std::string message(const std::string &msg);
    virtual void *getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify);
    virtual void memCopy(bh_view &src, bh_view &dst, const std::string &param);
    virtual void setMemoryPointer(bh_base *base, bool host_ptr, void *mem);
    virtual void *getDeviceContext();
    virtual void setDeviceContext(void *device_context);
    virtual std::string userKernel(const std::string &kernel, std::vector<bh_view> &operand_list,
                                   const std::string &compile_cmd, const std::string &tag, const std::string &param);
};

class ComponentImpl {
protected:
    // When disabled, a component passes everything through to its child.
    bool disabled = false;

public:
    // -1 is the bridge, 0 the first component of the stack list, ...
    const int stack_level;
    const ConfigParser config;
    ComponentFace child;

    explicit ComponentImpl(int stack_level, bool initiate_child = true)
        : stack_level(stack_level), config(stack_level) {
        init_child(initiate_child);
    }
    virtual ~ComponentImpl() = default;

    virtual void execute(BhIR *bhir) { child.execute(bhir); }
    virtual void extmethod(const std::string &name, bh_opcode opcode) { child.extmethod(name, opcode); }
    virtual std::string message(const std::string &msg) { return child.message(msg); }
    virtual void *getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify) {
        return child.getMemoryPointer(base, copy2host, force_alloc, nullify);
    }
    virtual void setMemoryPointer(bh_base *base, bool host_ptr, void *mem) {
        child.setMemoryPointer(base, host_ptr, mem);
    }
    virtual void memCopy(bh_view &src, bh_view &dst, const std::string &param) { child.memCopy(src, dst, param); }
    virtual void *getDeviceContext() { return child.getDeviceContext(); }
    virtual void setDeviceContext(void *device_context) { child.setDeviceContext(device_context); }
    virtual std::string userKernel(const std::string &kernel, std::vector<bh_view> &operand_list,
                                   const std::string &compile_cmd, const std::string &tag, const std::string &param) {
        return child.userKernel(kernel, operand_list, compile_cmd, tag, param);
    }

private:
    void init_child(bool initiate_child) {
        const std::string child_lib_path = config.getChildLibraryPath();
        if (initiate_child && !child_lib_path.empty()) {
            child = ComponentFace{child_lib_path, stack_level + 1};
        }
    }
};

// Base class of vector engines.
class ComponentVE : public ComponentImpl {
public:
    std::map<bh_opcode, extmethod::ExtmethodFace> extmethods;
    std::set<bh_opcode> child_extmethods;
    explicit ComponentVE(int stack_level, bool initiate_child = true) : ComponentImpl(stack_level, initiate_child) {}
};

} // namespace component
} // namespace bohrium
