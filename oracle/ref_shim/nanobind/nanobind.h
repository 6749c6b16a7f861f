// Minimal stand-in for the parts of nanobind that mach's kernel.cu names, so the
// unmodified reference source compiles into a plain shared library (the real
// nanobind is not installed in this image).  Written for this project; it only
// provides names and trivial bodies.
//
// Used solely to build the reference CUDA kernel under oracle/_ref/ as a
// checker and baseline.  Not part of the mach_b200 product.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

// ---- CPython warning API as used by src/mach/kernel.cu:357-423, 1092-1100 ----
using PyObject = void;
#define PyExc_RuntimeWarning (static_cast<PyObject*>(nullptr))
#define PyExc_UserWarning (static_cast<PyObject*>(nullptr))

// The last warning text the reference raised; read by the shim.
inline std::string& machref_warning_text() {
    static thread_local std::string msg;
    return msg;
}

inline int PyErr_WarnEx(PyObject*, const char* message, long) {
    machref_warning_text() = message ? message : "";
    return 0;
}

namespace nanobind {

namespace device {
struct cpu {
    static constexpr int32_t value = 1;
};
struct cuda {
    static constexpr int32_t value = 2;
};
}  // namespace device

template <size_t N>
struct ndim {};
template <long long... Dims>
struct shape {};
struct c_contig {};

// A borrowed view: pointer, shape and DLPack device type.  Shapes up to rank 4.
template <typename T, typename... Extra>
class ndarray {
public:
    ndarray() = default;
    ndarray(T* data, size_t rank, const size_t* dims, int32_t device_type)
        : data_(data), rank_(rank), device_type_(device_type) {
        for (size_t i = 0; i < rank && i < 4; ++i) dims_[i] = dims[i];
    }
    T* data() const { return data_; }
    size_t ndim() const { return rank_; }
    size_t shape(size_t i) const { return dims_[i]; }
    int32_t device_type() const { return device_type_; }
    size_t size() const {
        size_t n = 1;
        for (size_t i = 0; i < rank_; ++i) n *= dims_[i];
        return n;
    }
    size_t nbytes() const { return size() * sizeof(T); }

private:
    T* data_ = nullptr;
    size_t rank_ = 0;
    size_t dims_[4] = {0, 0, 0, 0};
    int32_t device_type_ = device::cpu::value;
};

struct arg {
    const char* name;
    arg noconvert() const { return *this; }
    template <typename V>
    arg operator=(V) const {
        return *this;
    }
};

namespace literals {
inline arg operator""_a(const char* s, size_t) { return arg{s}; }
}  // namespace literals

template <typename E>
struct enum_ {
    template <typename M>
    enum_(M&, const char*) {}
    enum_& value(const char*, E, const char* = nullptr) { return *this; }
    enum_& export_values() { return *this; }
};

}  // namespace nanobind

// The module body becomes an uninstantiated template: it is parsed but never run.
#define NB_MODULE(name, var) \
    template <typename NbModuleT> \
    [[maybe_unused]] static void machref_unused_module_##name(NbModuleT& var)
