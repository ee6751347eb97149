// diagnostics.h — drop-in for the reference's SimulationTiming / printDetailedTiming
// (diagnostics.h:5-61).  The compat step fills the fields with CUDA-event times (device
// time of each phase), not host clocks around asynchronous launches.
#pragma once
#include <iomanip>
#include <iostream>

struct SimulationTiming {
  double coordinate_update_us = 0.0;
  double collision_detection_us = 0.0;
  double particle_removal = 0.0;
  double density_reset_us = 0.0;
  double density_update_us = 0.0;
  double solver_us = 0.0;
  double electric_field_us = 0.0;
  double velocity_update_us = 0.0;
  double synchronize_us = 0.0;
  double mcc_us = 0.0;
  double total_us = 0.0;
};

inline void printDetailedTiming(const SimulationTiming& t, int steps, int particles) {
  std::cout << "\n=== DETAILED SIMULATION TIMING (microseconds) ===\n"
            << "Particles: " << particles << ", Steps: " << steps << "\n" << std::fixed << std::setprecision(2)
            << "  Particle pass:      " << t.coordinate_update_us / steps << " us\n"
            << "  Particle removal:   " << t.particle_removal / steps << " us\n"
            << "  Solver:             " << t.solver_us / steps << " us\n"
            << "  TOTAL:              " << t.total_us << " us\n"
            << "  Particles/us:       " << (double)particles * steps / t.total_us << "\n";
}
