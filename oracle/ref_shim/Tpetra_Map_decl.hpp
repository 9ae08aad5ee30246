// The ordinal and node typedefs of Tpetra::Map<> that the reference's
// Data/DefaultTypes.h reads (local ordinal int, global ordinal long long, the
// defaults of Trilinos 15), for the parity checker (oracle/_ref).  Test
// infrastructure only.
#pragma once

#include "Kokkos_Core.hpp"

namespace Tpetra {
struct HostNode {
    using execution_space = Kokkos::HostSpace;
    using memory_space = Kokkos::HostSpace;
};
template <class LO = int, class GO = long long, class Node = HostNode>
class Map {
public:
    using local_ordinal_type = LO;
    using global_ordinal_type = GO;
    using node_type = Node;
    using execution_space = typename Node::execution_space;
    using memory_space = typename Node::memory_space;
};
}  // namespace Tpetra
