// A view into a base array: start offset, shape and strides, all in elements.
// Fields, ordering operators and helpers follow include/bohrium/bh_view.hpp:45-219 and
// core/bh_view.cpp of the reference. A view whose base is nullptr stands for the
// instruction's constant operand.
#pragma once

#include <cassert>
#include <string>
#include <tuple>
#include <vector>
#include <bohrium/bh_static_vector.hpp>
#include <bohrium/bh_type.hpp>
#include <bohrium/bh_base.hpp>
#include <bohrium/bh_slide.hpp>

std::ostream &operator<<(std::ostream &out, const bh_base &b);

struct bh_view {
    bh_base *base = nullptr;
    int64_t start = 0;
    int64_t ndim = 0;
    BhIntVec shape;
    BhIntVec stride;
    bh_slide slides;

    bh_view() = default;
    bh_view(bh_base *base, int64_t start, int64_t ndim, BhIntVec shape, BhIntVec stride)
        : base(base), start(start), ndim(ndim), shape(std::move(shape)), stride(std::move(stride)) {}
    bh_view(const bh_view &view);
    bh_view &operator=(const bh_view &view) = default;
    // A contiguous 1-D view of the whole base.
    explicit bh_view(bh_base *b) : bh_view(b, 0, 1, {b->nelem()}, {1}) {}

    std::vector<std::tuple<int64_t, int64_t, int64_t>> python_notation() const;
    std::string pprint(bool python_notation = true) const;
    void insert_axis(int64_t dim, int64_t size, int64_t stride);
    void remove_axis(int64_t dim);
    void transpose(int64_t axis1, int64_t axis2);
    bool is_scalar() const { return shape.prod() == 1; }
    bool isConstant() const { return base == nullptr; }
    bool isContiguous() const;
    bool hasSlide() const { return !slides.dims.empty(); }

    bool operator<(const bh_view &other) const {
        if (base < other.base) return true;
        if (other.base < base) return false;
        if (start < other.start) return true;
        if (other.start < start) return false;
        if (ndim < other.ndim) return true;
        if (other.ndim < ndim) return false;
        for (int64_t i = 0; i < ndim; ++i) {
            if (shape[i] < other.shape[i]) return true;
            if (other.shape[i] < shape[i]) return false;
        }
        for (int64_t i = 0; i < ndim; ++i) {
            if (stride[i] < other.stride[i]) return true;
            if (other.stride[i] < stride[i]) return false;
        }
        return false;
    }
    bool operator==(const bh_view &other) const {
        if (base == nullptr || other.base == nullptr) return false;
        return base == other.base && ndim == other.ndim && start == other.start && shape == other.shape &&
               stride == other.stride;
    }
    bool operator!=(const bh_view &other) const { return !(*this == other); }
};

std::ostream &operator<<(std::ostream &out, const bh_view &v);

bool bh_view_same_shape(const bh_view *a, const bh_view *b);
// Two views are disjoint when they use different bases. Like the reference
// (core/bh_view.cpp:188-192), sharing a base is treated as overlapping.
bool bh_view_disjoint(const bh_view *a, const bh_view *b);
