// mcc.hpp — drop-in for the reference's MCC surface (mcc.hpp:6-21, mcc.cu:17-150).
#pragma once
#include <string>
#include <utility>
#include <vector>
#include "particles.cuh"

struct cross_sections {
  double* energies = nullptr;            // device arrays, as in the reference
  double* sigmas = nullptr;
  double* sigmas_elastic = nullptr;
  double* sigmas_ionization = nullptr;
  double* sigmas_excitation = nullptr;
  double* sigmas_recombination = nullptr;
  double* sigmas_attachment = nullptr;
  double* sigmas_transport = nullptr;
  int size = 0;
};

// Two-column text file (energy eV, sigma m^2), '#' comment lines skipped.
std::pair<std::vector<double>, std::vector<double>> read_cross_section(const std::string& filename);

// elasticCollisions (mcc.cu:114-150): P = 1 - exp(-density sigma(E) |v| dt) per particle with
// E = 1/2 m |v|^2 in eV (2D speed), isotropic 2D redirection keeping |v|.  Random numbers
// come from Philox-4x32-10 keyed by (seed, particle index, call count) instead of a
// time-seeded cuRAND generator, so calls are reproducible.
void elasticCollisions(Particles2D& particles, double density, double dt, cross_sections& crossections);
