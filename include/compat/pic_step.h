// pic_step.h — drop-in for the reference's updateSimulationCUDA (main.cu:37-140), which the
// reference defines in main.cu itself.  One call advances `steps` full PIC steps in the
// reference's order (drift, wall test + removal, CIC deposit, multigrid solve with the
// reference's settings, E field, gather + kick) in the reference's units
// (lap(phi) = sum q w, v += q/m E dt), walls = boundaries' segments.
#pragma once
#include "boundaries.h"
#include "diagnostics.h"
#include "grid.cuh"
#include "particles.cuh"

void updateSimulationCUDA(Particles2D& particles, Grid2D& grid, Boundaries2D& boundaries, int& step, double dt,
                          int steps, SimulationTiming& timing);
