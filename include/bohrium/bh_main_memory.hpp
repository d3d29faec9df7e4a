// Host memory of base arrays (include/bohrium/bh_main_memory.hpp of the reference):
// bh_data_malloc() gives a base host storage if it has none, bh_data_free() releases it.
#pragma once

#include <cstdint>
#include <bohrium/bh_base.hpp>

void bh_data_malloc(bh_base *base);
void bh_data_free(bh_base *base);
// Total and unused host memory in bytes (-1 if unknown).
int64_t bh_main_memory_total();
int64_t bh_main_memory_unused();
