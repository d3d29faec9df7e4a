// Extension-method plugins (include/bohrium/bh_extmethod.hpp:57-134 and core/bh_extmethod.cpp:33-101
// of the reference): an extmethod named N is found by searching the component's `libs` list for
// the C symbols N_create / N_destroy; its execute(instr, arg) runs one extension instruction.
#pragma once

#include <cassert>
#include <string>
#include <bohrium/bh_config_parser.hpp>
#include <bohrium/bh_instruction.hpp>

namespace bohrium {
namespace extmethod {

class ExtmethodImpl {
public:
    ExtmethodImpl() = default;
    virtual ~ExtmethodImpl() = default;
    // `arg` is component specific: the GPU engine passes itself, CPU engines pass nullptr.
    virtual void execute(bh_instruction *instr, void *arg) = 0;
};

class ExtmethodFace {
    std::string _name;
    void *_lib_handle = nullptr;
    ExtmethodImpl *(*_create)() = nullptr;
    void (*_destroy)(ExtmethodImpl *) = nullptr;
    ExtmethodImpl *_implementation = nullptr;

public:
    ExtmethodFace(const ConfigParser &parent_config, const std::string &name);
    ~ExtmethodFace();
    ExtmethodFace(ExtmethodFace &&other) noexcept
        : _name(std::move(other._name)), _lib_handle(other._lib_handle), _create(other._create),
          _destroy(other._destroy), _implementation(other._implementation) {
        other._lib_handle = nullptr;
        other._create = nullptr;
        other._destroy = nullptr;
        other._implementation = nullptr;
    }
    ExtmethodFace(const ExtmethodFace &) = delete;
    void execute(bh_instruction *instr, void *arg) {
        assert(_implementation != nullptr);
        _implementation->execute(instr, arg);
    }
    const std::string &name() const { return _name; }
};

class ExtmethodNotFound : public std::exception {
    std::string _msg;

public:
    explicit ExtmethodNotFound(std::string msg) : _msg(std::move(msg)) {}
    const char *what() const noexcept override { return _msg.c_str(); }
};

} // namespace extmethod
} // namespace bohrium
