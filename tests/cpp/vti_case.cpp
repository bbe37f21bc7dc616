// VTI output case, written once against the reference's interface: compiled
// with the reference's own headers it makes the golden files in
// tests/golden/vti/, compiled with the drop-in headers (m3lb_b200/facade) it
// must make the same bytes.
//
//   vti_case <outdir> <arrays.bin> [solver]
//
// arrays.bin: float32 values of a 5 x 4 x 3 grid -- 60 for "rho", 180 for
// "u", 60 for "chi".  Writes <outdir>/bin.vti (write_vti_bin, spacing pi/64),
// <outdir>/series.pvd (write_pvd) and, with "solver", <outdir>/rest.vti
// (write_vti of a D3Q27 BGK solver at rest, a solid row at y = 0).
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "collision/BGK.hpp"
#include "io/VtiWriter.hpp"
#include "memory/EsotericPull.hpp"
#include "solver/FluidSolver.hpp"

using namespace lbm;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string out = argv[1];
  std::vector<float> vals(300);
  {
    std::FILE* f = std::fopen(argv[2], "rb");
    if (!f || std::fread(vals.data(), sizeof(float), vals.size(), f) != vals.size()) return 3;
    std::fclose(f);
  }
  std::vector<VtiArray> arrays(3);
  arrays[0].name = "rho";
  arrays[0].ncomp = 1;
  arrays[0].data.assign(vals.begin(), vals.begin() + 60);
  arrays[1].name = "u";
  arrays[1].ncomp = 3;
  arrays[1].data.assign(vals.begin() + 60, vals.begin() + 240);
  arrays[2].name = "chi";
  arrays[2].ncomp = 1;
  arrays[2].data.assign(vals.begin() + 240, vals.end());
  write_vti_bin(out + "/bin.vti", 5, 4, 3, arrays, 3.14159265358979323846 / 64);
  write_pvd(out + "/series.pvd", {{0.0, "vti/f_0000.vti"},
                                   {0.1234567890123, "vti/f_0001.vti"},
                                   {2.5e-7, "f 2.vti"}});
  bool bad = false;
  try {
    write_vti_bin(out + "/never.vti", 5, 4, 2, arrays);
  } catch (const std::runtime_error& e) {
    bad = true;
    std::printf("%s\n", e.what());
  }
  if (!bad) return 4;
  if (argc > 3 && std::string(argv[3]) == "solver") {
    Kokkos::initialize(argc, argv);
    {
      using Coll = BGK<D3Q27, SecondOrderEquilibrium<D3Q27>, NoForcing, ShiftedPopulations>;
      Domain d(6, 5, 4, true, false, true);
      Coll c;
      c.omega = Real(1.25);
      FluidSolver<D3Q27, EsotericPull<D3Q27>, Coll> s(d, c);
      s.set_geometry([](Index, Index y, Index) -> CellType { return y == 0 ? Solid : Fluid; });
      s.initialize(Real(1));
      write_vti(out + "/rest.vti", s);
    }
    Kokkos::finalize();
  }
  return 0;
}
