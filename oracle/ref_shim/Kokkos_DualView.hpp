// Host-only DualView<T*> for the parity checker (oracle/_ref); see
// Kokkos_Core.hpp in this folder.  Host and device views are one array, so
// modify/sync are no-ops.
#pragma once

#include "Kokkos_Core.hpp"

namespace Kokkos {
template <class T>
class DualView;

template <class T>
class DualView<T*> {
public:
    using t_dev = View<T*>;
    using t_host = View<T*>;
    using host_mirror_space = HostSpace;
    using execution_space = HostSpace;
    using memory_space = HostSpace;

    DualView() = default;
    DualView(const std::string& label, std::size_t n) : d_view(label, n), h_view(d_view) {}
    void resize(std::size_t n) {
        d_view.resize_storage(n);
        h_view = d_view;
    }
    template <class Space>
    void modify() {}
    template <class Space>
    void sync() {}
    std::size_t extent(int) const { return h_view.size(); }

    t_dev d_view;
    t_host h_view;
};

template <class T>
void deep_copy(DualView<T*>& dst, const DualView<T*>& src) {
    deep_copy(dst.h_view, src.h_view);
}
}  // namespace Kokkos
