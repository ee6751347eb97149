// grid.cuh — drop-in for the reference's Grid2D (grid.cuh:7-24, grid.cu:10-53).
// rho, phi (FP64) and E (double2, E = -grad phi) are device arrays of m*n nodes, row-major
// j*m + i.  Unlike the reference they start zeroed, so phi's boundary (the Dirichlet data of
// the field solve) is 0 until the caller writes it.  updateSimulationCUDA refreshes all three.
#pragma once
#include <cuda_runtime.h>

class Grid2D {
 public:
  double* rho = nullptr;
  double* phi = nullptr;
  double2* E = nullptr;
  int m = 0;
  int n = 0;
  double dx = 0.0;
  double dy = 0.0;
  double x = 0.0;
  double y = 0.0;

  Grid2D(int M, int N, double X, double Y);
  ~Grid2D();
  Grid2D(const Grid2D&) = delete;
  Grid2D& operator=(const Grid2D&) = delete;
  void debugGrid();
};
