// A Bohrium base array: element count, element type and the host data pointer.
// Fields and accessors follow include/bohrium/bh_base.hpp:30-98 of the reference.
#pragma once

#include <string>
#include <bohrium/bh_type.hpp>
#include <bohrium/bh_constant.hpp>

struct bh_base {
private:
    int64_t _nelem = 0;
    bh_type _type = bh_type::BOOL;
    void *_data = nullptr;

public:
    bh_base() = default;
    bh_base(int64_t nelem, bh_type type, void *data = nullptr) : _nelem(nelem), _type(type), _data(data) {}

    int64_t nelem() const noexcept { return _nelem; }
    bh_type dtype() const noexcept { return _type; }
    void *getDataPtr() { return _data; }
    const void *getDataPtr() const { return _data; }
    void resetDataPtr(void *data_ptr = nullptr) { _data = data_ptr; }
    // Unique label used in pretty printing (the address, like the reference's getLabel()).
    uint64_t getLabel() const;
    std::string str() const;
    int64_t nbytes() const { return nelem() * bh_type_size(_type); }
};
