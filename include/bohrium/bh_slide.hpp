// Sliding-view description used by do_while loops (flush-and-repeat).
// Fields follow include/bohrium/bh_slide.hpp:29-101 of the reference.
#pragma once

#include <cstdint>
#include <map>
#include <utility>
#include <vector>

struct bh_slide_dim {
    int64_t rank;          // the sliding dimension
    int64_t offset_change; // offset change per iteration (in units of `stride`)
    int64_t shape_change;  // shape change per iteration
    int64_t stride;        // stride of the sliding dimension
    int64_t shape;         // shape of the dimension (wrap-around of negative indices)
    int64_t step_delay;    // slide only every `step_delay` iterations
};

struct bh_slide {
    std::vector<bh_slide_dim> dims;
    int64_t iteration_counter = 0;
    // dimension -> (reset after this many slides, offset change accumulated since the last reset)
    std::map<int64_t, std::pair<int64_t, int64_t>> resets;

    void transpose(int64_t axis1, int64_t axis2) {
        for (bh_slide_dim &dim : dims) {
            if (dim.rank == axis1) {
                dim.rank = axis2;
            } else if (dim.rank == axis2) {
                dim.rank = axis1;
            }
        }
        auto a1 = resets.find(axis1);
        auto a2 = resets.find(axis2);
        if (a1 != resets.end() && a2 != resets.end()) {
            std::swap(a1->second, a2->second);
        } else if (a1 != resets.end()) {
            resets[axis2] = a1->second;
            resets.erase(a1);
        } else if (a2 != resets.end()) {
            resets[axis1] = a2->second;
            resets.erase(a2);
        }
    }
};
