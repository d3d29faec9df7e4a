// Host storage of base arrays (core/bh_main_memory.cpp:59-132 of the reference uses mmap; this
// uses 64-byte aligned heap blocks, which host<->device copies handle equally well).
#include <cstdlib>
#include <cstring>
#include <new>
#include <unistd.h>
#include <bohrium/bh_main_memory.hpp>

void bh_data_malloc(bh_base *base) {
    if (base == nullptr || base->getDataPtr() != nullptr) return;
    const int64_t nbytes = base->nbytes();
    if (nbytes <= 0) return;
    void *p = nullptr;
    const size_t sz = (static_cast<size_t>(nbytes) + 63) / 64 * 64;
    if (posix_memalign(&p, 64, sz) != 0 || p == nullptr) throw std::bad_alloc();
    base->resetDataPtr(p);
}

void bh_data_free(bh_base *base) {
    if (base == nullptr) return;
    free(base->getDataPtr());
    base->resetDataPtr(nullptr);
}

int64_t bh_main_memory_total() {
    const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
    return pages > 0 && page > 0 ? static_cast<int64_t>(pages) * page : -1;
}

int64_t bh_main_memory_unused() {
    const long pages = sysconf(_SC_AVPHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
    return pages > 0 && page > 0 ? static_cast<int64_t>(pages) * page : -1;
}
