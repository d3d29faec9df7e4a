// Fixed-capacity vector used for view shapes and strides.
//
// Interface follows include/bohrium/bh_static_vector.hpp of the reference (BhStaticVector /
// BhIntVec with capacity BH_MAXDIM = 16, plus sum()/prod()/pprint()). The reference derives from
// boost::container::static_vector and declares those helpers virtual; this version is a plain
// aggregate with inline storage and no vtable, so it is source compatible but not binary
// compatible with a reference build.
#pragma once

#include <cstdint>
#include <cstddef>
#include <initializer_list>
#include <numeric>
#include <functional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <ostream>

constexpr int64_t BH_MAXDIM = 16;

template <typename T>
class BhStaticVector {
    T _data[BH_MAXDIM];
    size_t _size = 0;

public:
    using value_type = T;
    using iterator = T *;
    using const_iterator = const T *;

    BhStaticVector() = default;
    explicit BhStaticVector(size_t n, const T &v = T{}) { resize(n, v); }
    BhStaticVector(std::initializer_list<T> l) {
        for (const T &v : l) push_back(v);
    }
    template <typename It, typename = decltype(*std::declval<It>())>
    BhStaticVector(It first, It last) {
        for (; first != last; ++first) push_back(static_cast<T>(*first));
    }

    size_t size() const noexcept { return _size; }
    bool empty() const noexcept { return _size == 0; }
    static constexpr size_t capacity() noexcept { return BH_MAXDIM; }
    T *data() noexcept { return _data; }
    const T *data() const noexcept { return _data; }
    iterator begin() noexcept { return _data; }
    iterator end() noexcept { return _data + _size; }
    const_iterator begin() const noexcept { return _data; }
    const_iterator end() const noexcept { return _data + _size; }
    T &operator[](size_t i) noexcept { return _data[i]; }
    const T &operator[](size_t i) const noexcept { return _data[i]; }
    T &at(size_t i) {
        if (i >= _size) throw std::out_of_range("BhStaticVector::at");
        return _data[i];
    }
    const T &at(size_t i) const {
        if (i >= _size) throw std::out_of_range("BhStaticVector::at");
        return _data[i];
    }
    T &front() { return _data[0]; }
    T &back() { return _data[_size - 1]; }
    const T &front() const { return _data[0]; }
    const T &back() const { return _data[_size - 1]; }

    void push_back(const T &v) {
        if (_size >= BH_MAXDIM) throw std::length_error("BhStaticVector: more than BH_MAXDIM elements");
        _data[_size++] = v;
    }
    void pop_back() { --_size; }
    void clear() noexcept { _size = 0; }
    void resize(size_t n, const T &v = T{}) {
        if (n > BH_MAXDIM) throw std::length_error("BhStaticVector: more than BH_MAXDIM elements");
        for (size_t i = _size; i < n; ++i) _data[i] = v;
        _size = n;
    }
    iterator insert(const_iterator pos, const T &v) {
        const size_t idx = static_cast<size_t>(pos - _data);
        if (_size >= BH_MAXDIM) throw std::length_error("BhStaticVector: more than BH_MAXDIM elements");
        for (size_t i = _size; i > idx; --i) _data[i] = _data[i - 1];
        _data[idx] = v;
        ++_size;
        return _data + idx;
    }
    iterator erase(const_iterator pos) {
        const size_t idx = static_cast<size_t>(pos - _data);
        for (size_t i = idx; i + 1 < _size; ++i) _data[i] = _data[i + 1];
        --_size;
        return _data + idx;
    }

    T sum() const { return std::accumulate(begin(), end(), T{0}); }
    T prod() const { return std::accumulate(begin(), end(), T{1}, std::multiplies<T>()); }
    std::string pprint() const {
        std::stringstream ss;
        ss << '(';
        for (size_t i = 0; i < _size; ++i) {
            if (i) ss << ',';
            ss << _data[i];
        }
        ss << ')';
        return ss.str();
    }

    bool operator==(const BhStaticVector &o) const {
        if (_size != o._size) return false;
        for (size_t i = 0; i < _size; ++i)
            if (!(_data[i] == o._data[i])) return false;
        return true;
    }
    bool operator!=(const BhStaticVector &o) const { return !(*this == o); }
    bool operator<(const BhStaticVector &o) const {
        const size_t n = _size < o._size ? _size : o._size;
        for (size_t i = 0; i < n; ++i) {
            if (_data[i] < o._data[i]) return true;
            if (o._data[i] < _data[i]) return false;
        }
        return _size < o._size;
    }
};

template <typename T>
inline std::ostream &operator<<(std::ostream &o, const BhStaticVector<T> &vec) {
    return o << vec.pprint();
}

typedef BhStaticVector<int64_t> BhIntVec;
