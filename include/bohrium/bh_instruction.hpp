// A Bohrium instruction (one bytecode).
// Fields and methods follow include/bohrium/bh_instruction.hpp:36-177 and
// core/bh_instruction.cpp of the reference.
#pragma once

#include <set>
#include <string>
#include <vector>
#include <bohrium/bh_opcode.h>
#include <bohrium/bh_view.hpp>
#include <bohrium/bh_constant.hpp>

// Iterable range over the non-constant operands of an instruction (the reference returns a
// boost::filtered_range with the same meaning).
template <typename Vec, typename View>
class bh_view_range {
    Vec *_ops;

public:
    class iterator {
        Vec *_ops;
        size_t _i;
        void skip() {
            while (_i < _ops->size() && (*_ops)[_i].isConstant()) ++_i;
        }

    public:
        iterator(Vec *ops, size_t i) : _ops(ops), _i(i) { skip(); }
        View &operator*() const { return (*_ops)[_i]; }
        View *operator->() const { return &(*_ops)[_i]; }
        iterator &operator++() {
            ++_i;
            skip();
            return *this;
        }
        bool operator!=(const iterator &o) const { return _i != o._i; }
        bool operator==(const iterator &o) const { return _i == o._i; }
    };
    explicit bh_view_range(Vec *ops) : _ops(ops) {}
    iterator begin() const { return iterator(_ops, 0); }
    iterator end() const { return iterator(_ops, _ops->size()); }
    bool empty() const { return !(begin() != end()); }
};

struct bh_instruction {
    bh_opcode opcode = -1;
    std::vector<bh_view> operand;
    bh_constant constant{};
    // Set when the instruction creates (first writes) its output array.
    bool constructor = false;
    // Identifies the original instruction across reshape/transpose/copy transformations.
    int64_t origin_id = -1;

    bh_instruction() = default;
    bh_instruction(bh_opcode opcode, std::vector<bh_view> operands) : opcode(opcode), operand(std::move(operands)) {}
    bh_instruction(const bh_instruction &instr) = default;
    bh_instruction &operator=(const bh_instruction &instr) = default;

    std::set<bh_base *> get_bases();
    bh_view_range<std::vector<bh_view>, bh_view> getViews() { return bh_view_range<std::vector<bh_view>, bh_view>(&operand); }
    bh_view_range<const std::vector<bh_view>, const bh_view> getViews() const {
        return bh_view_range<const std::vector<bh_view>, const bh_view>(&operand);
    }
    bool has_constant() const {
        for (const bh_view &v : operand)
            if (v.isConstant()) return true;
        return false;
    }
    bool isContiguous() const;
    bool all_same_shape() const;
    bool reshapable() const;
    // The principal shape: the shape of the computation (the input shape for sweeps).
    BhIntVec shape() const;
    int64_t ndim() const;
    // The swept axis of a reduction/accumulate, BH_MAXDIM otherwise.
    int sweep_axis() const;
    void reshape(const std::vector<int64_t> &shape);
    void remove_axis(int64_t axis);
    void transpose(int64_t axis1, int64_t axis2);
    void transpose();
    bh_type operand_type(int operand_index) const;
    std::string pprint(bool python_notation = true) const;

    bool operator==(const bh_instruction &other) const {
        if (opcode != other.opcode || operand.size() != other.operand.size()) return false;
        for (size_t i = 0; i < operand.size(); ++i) {
            if (operand[i].isConstant() != other.operand[i].isConstant()) return false;
            if (operand[i].isConstant()) {
                if (constant != other.constant) return false;
            } else if (operand[i] != other.operand[i]) {
                return false;
            }
        }
        return true;
    }
    bool operator!=(const bh_instruction &other) const { return !(*this == other); }
};

std::ostream &operator<<(std::ostream &out, const bh_instruction &instr);

// True when `b` must run after `a` (they share a base and one of them writes it).
bool bh_instr_dependency(const bh_instruction *a, const bh_instruction *b);
