// A caller written against the reference's IMEXRK surface, as its
// executables use it (StateVector::FixedEvolve, StateVector.cpp:85-105:
// set dt, UpdateForTimestep, FilterAll, PopulateNodalVariables,
// RemoveDivergence(0), then TimeStep in a loop), compiled against the drop-in
// header stratiflow_b200/host/imexrk.hpp. The grid is the reduced 3D shear
// layer 64 x 32 x 64.
//
//   dropin_fixed_evolve IN OUT NSTEPS
// IN:  L1 L2 L3 Re Ri Pr dt (7 doubles), U[N3], dB/dz[N3] (doubles), then
//      u1, u2, u3, b, p as complex<float> in the reference layout
// OUT: u1, u2, u3, b, p after NSTEPS steps, then KE, PE (doubles)
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../stratiflow_b200/host/imexrk.hpp"

using namespace stratiflow;
constexpr int N1 = 64, N2 = 32, N3 = 64;

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s IN OUT NSTEPS\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  double prm[7];
  std::vector<double> U(N3), dB(N3);
  if (std::fread(prm, sizeof(double), 7, in) != 7) return 2;
  if (std::fread(U.data(), sizeof(double), N3, in) != (size_t)N3) return 2;
  if (std::fread(dB.data(), sizeof(double), N3, in) != (size_t)N3) return 2;
  FlowParams fp;
  fp.L1 = prm[0]; fp.L2 = prm[1]; fp.L3 = prm[2]; fp.Re = prm[3]; fp.Ri = prm[4]; fp.Pr = prm[5];
  try {
    IMEXRK<N1, N2, N3> solver(fp);
    for (auto* m : {&solver.u1, &solver.u2, &solver.u3, &solver.b, &solver.p})
      if (std::fread(m->Raw(), sizeof(std::complex<float>), m->size(), in) != m->size()) return 2;
    std::fclose(in);
    IMEXRK<N1, N2, N3>::Neumann1D Ubar(BoundaryCondition::Neumann);
    for (int k = 0; k < N3; k++) Ubar(k) = U[k];
    solver.SetStratification(dB);
    solver.SetBackground(Ubar);
    // FixedEvolve (StateVector.cpp:85-105)
    solver.deltaT = (stratifloat)prm[6];
    solver.UpdateForTimestep();
    solver.FilterAll();
    solver.PopulateNodalVariables();
    solver.RemoveDivergence(0.0);
    const int nsteps = std::atoi(argv[3]);
    for (int step = 0; step < nsteps; step++) solver.TimeStep();
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    for (auto* m : {&solver.u1, &solver.u2, &solver.u3, &solver.b, &solver.p})
      std::fwrite(m->Raw(), sizeof(std::complex<float>), m->size(), out);
    const double e[2] = {solver.KE(), solver.PE()};
    std::fwrite(e, sizeof(double), 2, out);
    std::fclose(out);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "%s\n", ex.what());
    return 1;
  }
  return 0;
}
