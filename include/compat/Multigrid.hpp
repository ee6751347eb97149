// Multigrid.hpp — drop-in for the reference's solver entry point (Multigrid.hpp:3-11).
// Solves lap(phi) = rho in place on caller-owned FP64 device arrays (boundary values of phi
// are the Dirichlet data, phi is the warm start) with the reference's V-cycle: red-black SOR
// with omega, 3 pre / 3 post sweeps, 20 on the coarsest of `levels` levels, V-cycles until
// ||rho - lap(phi)|| / ||rho|| < 1e-5 or 50 cycles.  Runs on the engine's FP32 V-cycles inside
// FP64 defect correction.
#pragma once

void solve_multigrid(double* phi_d, double* rho_d, int nx, int ny, int levels, double h, double omega = 1.25);
