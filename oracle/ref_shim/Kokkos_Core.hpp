// Host-only stand-in for the few Kokkos types the reference's GridVector,
// MatrixBlock and BiCGStab2 headers name (View<T*>, DualView<T*>, deep_copy),
// so that those headers compile unmodified into the parity checker
// (oracle/_ref).  Test
// infrastructure only.  A View is a reference-counted host array; a DualView
// holds one such array as both its host and its device view.
#pragma once

#include <cstddef>
#include <memory>
#include <string>
#include <vector>

namespace Kokkos {
struct HostSpace {
    using execution_space = HostSpace;
    using memory_space = HostSpace;
};
using DefaultExecutionSpace = HostSpace;
using DefaultHostExecutionSpace = HostSpace;

template <class T, class... Props>
class View;

template <class T, class... Props>
class View<T*, Props...> {
public:
    using value_type = T;
    View() : v(std::make_shared<std::vector<T>>()) {}
    View(const std::string& label, std::size_t n) : lbl(label), v(std::make_shared<std::vector<T>>(n)) {}
    T& operator[](std::size_t i) const { return (*v)[i]; }
    T& operator()(std::size_t i) const { return (*v)[i]; }
    std::size_t size() const { return v->size(); }
    std::size_t extent(int) const { return v->size(); }
    T* data() const { return v->data(); }
    const std::string& label() const { return lbl; }
    void resize_storage(std::size_t n) { v->resize(n); }

private:
    std::string lbl;
    std::shared_ptr<std::vector<T>> v;
};

template <class T, class... P, class... Q>
void deep_copy(const View<T*, P...>& dst, const View<T*, Q...>& src) {
    for (std::size_t i = 0; i < src.size() && i < dst.size(); i++) dst[i] = src[i];
}
template <class T, class... P>
void deep_copy(const View<T*, P...>& dst, const T& value) {
    for (std::size_t i = 0; i < dst.size(); i++) dst[i] = value;
}
}  // namespace Kokkos
