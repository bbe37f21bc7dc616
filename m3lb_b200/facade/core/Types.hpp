// Scalar types, container aliases and execution spaces of the B200 drop-in
// (the names of src/core/Types.hpp).  Real is the host-side precision of the
// API (parameters, returned fields); the device storage precision is chosen
// per solver (solver/FluidSolver.hpp).
#pragma once
#include <cstdint>
#include <utility>

#include "Kokkos_Core.hpp"

namespace lbm {

#if defined(LBM_SINGLE_PRECISION)
using Real = float;
#else
using Real = double;
#endif

inline constexpr const char* precision_name() { return sizeof(Real) == 4 ? "FP32" : "FP64"; }

using Index = std::int32_t;

using ExecSpace = Kokkos::DefaultExecutionSpace;
using MemSpace = ExecSpace::memory_space;
using HostSpace = Kokkos::DefaultHostExecutionSpace;

template <class T> using View1D = Kokkos::View<T*, MemSpace>;
template <class T> using View2D = Kokkos::View<T**, MemSpace>;
template <class V> using MirrorOf = decltype(Kokkos::create_mirror_view(std::declval<V>()));
template <class T> using HostView1D = MirrorOf<View1D<T>>;
template <class T> using HostView2D = MirrorOf<View2D<T>>;

using Range = Kokkos::RangePolicy<ExecSpace>;

}  // namespace lbm
