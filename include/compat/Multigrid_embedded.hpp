// Multigrid_embedded.hpp — drop-in for the reference's embedded-boundary solver class
// (Multigrid_embedded.cu:106-190; the reference defines MGLevel and Multigrid in that .cu file
// and ships no header for them).  Same members, constructor arguments and vcycle(l): level l
// holds nx*ny FP64 phi / rhs / res / phi_bc and a node-kind mask (FLUID 0, DIRICHLET 1,
// SOLID 2), sizes (n-1)/2+1 per level, all zeroed at construction; the caller fills
// levels[0].phi, rhs, mask and phi_bc and calls vcycle(0) as often as it likes.
// vcycle runs the B200 kernels of pic_solve_embedded_f64 with the reference's operators
// (2 + 2 red-black Gauss-Seidel sweeps, coarse kind injected from (2i, 2j), prolongation from
// (i/2, j/2)) on the legacy default stream, like the reference.  Differences, deliberate:
//   * the second colour of each sweep updates the odd nodes only (the reference's colour
//     test, :22, lets it update every node at once);
//   * res is not written (the residual is formed inside the restriction);
//   * the class is non-copyable and errors throw std::runtime_error.
#pragma once
#include <vector>

#ifndef FLUID
#define FLUID 0
#endif
#ifndef DIRICHLET
#define DIRICHLET 1
#endif
#ifndef SOLID
#define SOLID 2
#endif

struct MGLevel {
  int nx, ny;
  double *phi, *rhs, *res;
  unsigned char* mask;
  double* phi_bc;
};

class Multigrid {
 public:
  std::vector<MGLevel> levels;
  double h;
  int max_levels;

  Multigrid(int nx, int ny, int levels_in, double h_in);
  ~Multigrid();
  Multigrid(const Multigrid&) = delete;
  Multigrid& operator=(const Multigrid&) = delete;
  void vcycle(int l);

 private:
  std::vector<double*> alt_;   // second phi buffer per level (tile kernels never write in place)
};
