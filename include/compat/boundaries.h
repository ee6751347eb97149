// boundaries.h — drop-in for the reference's Boundaries2D (boundaries.h:7-23,
// boundaries.cu:3-25).  Walls are segments in domain units; a particle whose drift crosses
// one is removed by updateSimulationCUDA.  At most 64 walls.
#pragma once
#include <cuda_runtime.h>
#include <vector>

class Boundaries2D {
 public:
  Boundaries2D(int width, int height, int nx, int ny) : width(width), height(height), nx(nx), ny(ny) {}
  ~Boundaries2D();
  Boundaries2D(const Boundaries2D&) = delete;
  Boundaries2D& operator=(const Boundaries2D&) = delete;
  void add_wall(double x1, double y1, double x2, double y2);
  // Uploads the walls to d_walls (double4) and d_walls_int (int4, truncated), as the reference.
  void compile_walls();
  int wall_count = 0;
  std::vector<double> walls;  // x1, y1, x2, y2 per wall
  double4* d_walls = nullptr;
  int4* d_walls_int = nullptr;

 private:
  int width, height;
  int nx, ny;
};
