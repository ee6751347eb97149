// particles.cuh — drop-in for the reference's Particles2D (particles.cuh:3-39,
// particles.cu:112-262).
//
// r, r_old, v (double2) and type (int) are device arrays the caller writes with cudaMemcpy,
// exactly as the reference's main.cu:232-238 does, and last_alive is the live count.  The
// species tables q, m are device arrays; species 0 starts as q = 0.1, m = 1.0
// (particles.cu:146-149).  v_abs, energy and crs are filled by elasticCollisions.
// collided_indices / collision_counter hold the particles removed by the last
// updateSimulationCUDA call, as indices into the arrays as they were when that call began
// (for one step per call, the reference's hit list).
//
// The reference's removal scratch (swap_counter, d_last_alive, d_collision_flags,
// d_count_head/tail, d_remove_in_head, d_stay_in_tail, h_current_stamp, ionization_flags)
// has no counterpart: removal here is a stable compaction with its own scratch.
// Errors (allocation, bad species, engine failures) throw std::runtime_error.
#pragma once
#include <cuda_runtime.h>

class Grid2D;
class Boundaries2D;
struct SimulationTiming;
struct cross_sections;
namespace pic_compat {
struct State;
}

class Particles2D {
 public:
  int max_particles = 0;
  double2* r = nullptr;
  double2* r_old = nullptr;  // positions before the last drift
  double2* v = nullptr;
  double* v_abs = nullptr;
  double* energy = nullptr;
  double* crs = nullptr;
  int* type = nullptr;
  double* q = nullptr;
  double* m = nullptr;
  int* collided_indices = nullptr;
  int* collision_counter = nullptr;
  int last_alive = 0;

  explicit Particles2D(const int num_particles);
  ~Particles2D();
  Particles2D(const Particles2D&) = delete;
  Particles2D& operator=(const Particles2D&) = delete;
  void add_species(double m, double q);  // argument order (m, q) as in the reference
  void change_species(int species, double m, double q);
  void debugParticles(int num_to_print = 5);
  // Removes the particles listed in collided_indices[0 .. *collision_counter) and keeps
  // the others in their order (indices outside [0, last_alive) and repeats are ignored).
  void removeCollidedParticles();
  int species_count() const { return species_num; }

 private:
  int species_num = 1;
  pic_compat::State* state_ = nullptr;  // engine job, scratch, random stream counter
  friend void updateSimulationCUDA(Particles2D&, Grid2D&, Boundaries2D&, int&, double, int, SimulationTiming&);
  friend void elasticCollisions(Particles2D&, double, double, cross_sections&);
};
