// kernels.cuh — the reference's per-kernel entry points (kernels.cuh:14-77, kernels.cu),
// as host functions with the same names and arguments plus an optional stream.  Each
// launches one kernel on FP64 AoS device arrays with the reference's arithmetic:
//   update_coordinates          r_old <- r; r <- r + v dt                  (kernels.cu:8-23)
//   updateDensity               rho += q[type] * CIC weights, skip outside (kernels.cu:26-69)
//   updateParticleVelocities    v += q/m E_CIC(r) dt, skip outside         (kernels.cu:71-131)
//   computeElectricField        E = -grad(phi), central inside, one-sided on edges (kernels.cu:134-191)
//   compute_speeds_and_energies |v| and 1/2 m |v|^2 * 6.25e18 eV          (kernels.cu:196-215)
//   interpolate_cross_sections  linear in energy, clipped at the ends      (kernels.cu:219-263)
//   convertPositionsToFloat     double2 -> float2                          (kernels.cu:268-274)
// The caller's launch configuration is not needed: each call covers all elements.
#pragma once
#include <cuda_runtime.h>

void update_coordinates(double2* positions_new, double2* positions_old, const double2* velocities,
                        const int num_particles, const double dt, cudaStream_t stream = 0);
void updateDensity(double* d_rho, const double2* d_positions, const double* d_q_type, const int* d_part_type, int m,
                   int n, double dx, double dy, int last_alive, cudaStream_t stream = 0);
void updateParticleVelocities(double2* velocities, const double2* E_grid, const double2* positions,
                              const int* part_types, const double* charge, const double* mass, int num_particles,
                              double dx, double dy, int m, int n, double dt, cudaStream_t stream = 0);
void computeElectricField(double2* E_grid, const double* phi, int m, int n, double dx, double dy,
                          cudaStream_t stream = 0);
void compute_speeds_and_energies(const double2* V, double* V_abs, double* energies, const int* type_arr,
                                 const double* m_type, const int N, cudaStream_t stream = 0);
void interpolate_cross_sections(const double* energies, const double* xs_energy, const double* xs_values,
                                double* output, const int xs_len, const int N, cudaStream_t stream = 0);
void convertPositionsToFloat(const double2* d_positions, float2* f_positions, int count, cudaStream_t stream = 0);
