// collisions.cuh — the reference's wall test (collisions.cuh:4-12, collisions.cu:7-54) as a
// host function: appends to collided_indices the index of every particle whose move
// p0 -> p1 crosses one of the walls (x1, y1, x2, y2), counting in *collision_counter.
// The order of the list is unspecified (atomic append), as in the reference.  Parallel
// moves are recognised by an exact zero determinant rather than the reference's absolute
// 1e-10 cut-off, which also discards slow, non-parallel crossings.
#pragma once
#include <cuda_runtime.h>

void detect_intersections(const double2* p0, const double2* p1, const double4* walls, int* collided_indices,
                          int* collision_counter, const int num_particles, const int num_walls,
                          cudaStream_t stream = 0);
