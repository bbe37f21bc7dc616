// One slice of the reference-solver instantiations, selected by macros so the
// slices compile in parallel (see oracle/Makefile).  REF_LAT is D2Q9 or D3Q27,
// REF_STRM EsotericPull or TwoLattice, REF_FORCE Guo or NoForcing, REF_STORE
// ShiftedPopulations or RawPopulations, REF_NAME the exported factory name.
#include "ref_impl.hpp"

namespace refdrv {
Base* REF_NAME(int op, int eq, const Domain& d, const Params& p) {
  using L = lbm::REF_LAT;
  using Strm = lbm::REF_STRM<L>;
  using F = lbm::REF_FORCE;
  using S = lbm::REF_STORE;
  using E2 = SecondOrderEquilibrium<L>;
  using EP = ProductFormEquilibrium<L>;
  switch (op) {
    case 0: return new Impl<L, Strm, NoCollision<L>>(d, p);
    case 1: return eq ? (Base*)new Impl<L, Strm, BGK<L, EP, F, S>>(d, p)
                      : (Base*)new Impl<L, Strm, BGK<L, E2, F, S>>(d, p);
    case 2: return eq ? (Base*)new Impl<L, Strm, TRT<L, EP, F, S>>(d, p)
                      : (Base*)new Impl<L, Strm, TRT<L, E2, F, S>>(d, p);
    case 3: return new Impl<L, Strm, MomentCollision<L, F, S, false>>(d, p);
    case 4: return new Impl<L, Strm, MomentCollision<L, F, S, true>>(d, p);
    default: return nullptr;
  }
}
}  // namespace refdrv
