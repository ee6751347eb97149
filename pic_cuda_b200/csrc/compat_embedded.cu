// compat_embedded.cu — the reference's embedded-boundary Multigrid class
// (Multigrid_embedded.cu:106-190) on the kernels of mg_embedded.cu.
#include <stdexcept>
#include <string>
#include "../../include/compat/Multigrid_embedded.hpp"
#include "kernels.h"

namespace {
[[noreturn]] void raise(const std::string& what) { throw std::runtime_error("pic compat: " + what); }
void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) raise(std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

// Multigrid::Multigrid (Multigrid_embedded.cu:119-146): every level's arrays allocated and
// zeroed; level sizes (n - 1) / 2 + 1.
Multigrid::Multigrid(int nx, int ny, int levels_in, double h_in) : h(h_in), max_levels(levels_in) {
  if (nx < 3 || ny < 3 || levels_in < 1 || levels_in > PIC_MAX_LEVELS || !(h_in > 0))
    raise("Multigrid: needs nx, ny >= 3, 1..14 levels and h > 0");
  int nxf = nx, nyf = ny;
  for (int l = 0; l < levels_in; ++l) {
    MGLevel L{};
    L.nx = nxf; L.ny = nyf;
    const size_t N = (size_t)nxf * nyf;
    double* alt = nullptr;
    ck(cudaMalloc(&L.phi, N * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc(&L.rhs, N * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc(&L.res, N * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc(&L.mask, N), "cudaMalloc");
    ck(cudaMalloc(&L.phi_bc, N * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc(&alt, N * sizeof(double)), "cudaMalloc");
    ck(cudaMemset(L.phi, 0, N * sizeof(double)), "cudaMemset");
    ck(cudaMemset(L.rhs, 0, N * sizeof(double)), "cudaMemset");
    ck(cudaMemset(L.res, 0, N * sizeof(double)), "cudaMemset");
    ck(cudaMemset(L.mask, 0, N), "cudaMemset");
    ck(cudaMemset(L.phi_bc, 0, N * sizeof(double)), "cudaMemset");
    levels.push_back(L);
    alt_.push_back(alt);
    nxf = (nxf - 1) / 2 + 1;
    nyf = (nyf - 1) / 2 + 1;
  }
}

Multigrid::~Multigrid() {
  for (auto& L : levels) {
    cudaFree(L.phi); cudaFree(L.rhs); cudaFree(L.res); cudaFree(L.mask); cudaFree(L.phi_bc);
  }
  for (double* p : alt_) cudaFree(p);
}

// Multigrid::vcycle (Multigrid_embedded.cu:159-188) from level l.
void Multigrid::vcycle(int l) {
  if (l < 0 || l >= max_levels) raise("vcycle: level out of range");
  EmbLevels P;
  emb_layout(P, levels[0].nx, levels[0].ny, max_levels);
  for (int k = 0; k < max_levels; ++k) {
    P.phi[k] = levels[k].phi;
    P.alt[k] = alt_[k];
    P.rhs[k] = levels[k].rhs;
    P.mask[k] = levels[k].mask;
    P.bc[k] = levels[k].phi_bc;
  }
  P.h = h;
  if (emb_vcycle(P, l, 2, 2, 0, 0) != PIC_OK) raise(std::string("vcycle: ") + pic_last_error());
}
