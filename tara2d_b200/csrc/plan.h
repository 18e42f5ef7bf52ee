// Host side of a grid: sizes, read-only device tables and error handling.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "spectral.cuh"
#include "prof.h"
#include "../../include/tara2d_gpu.h"

namespace tara {

// Last error text of the calling thread (tara_last_error()).
void set_error(const std::string& msg);
const char* last_error();

#define TARA_CUDA_TRY(expr)                                                           \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      ::tara::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));          \
      return TARA_ECUDA;                                                              \
    }                                                                                 \
  } while (0)

#define TARA_TRY(expr)                  \
  do {                                  \
    int s_ = (expr);                    \
    if (s_ != TARA_OK) return s_;       \
  } while (0)

bool supported_length(int n);

// e^{-2 pi i m / L} with octant reduction, exact at multiples of pi/4.
void twiddle(long m, long L, long double& c, long double& s);

// Wavenumbers and the dealiasing cut-off with the reference's FP64 formulas
// (src/derive2coh.f95:58-86 for k, :208-212 for the circular 2/3 rule).
void wavenumbers(int Nx, int Ny, double Lx, double Ly, double pi, std::vector<double>& kx,
                 std::vector<double>& ky, std::vector<int>& cut);

template <class T>
struct Grid {
  int Nx = 0, Ny = 0, Nh = 0, ld = 0;
  double Lx = 0, Ly = 0, pi = 0;
  Tables<T> tb{};
  Prof* prof = nullptr;  // per-kernel timing (owned by the session)
  void* dmem = nullptr;  // one allocation for all tables
  size_t field_elems() const { return (size_t)Ny * ld; }
  size_t field_bytes() const { return field_elems() * sizeof(Cx<T>); }
  int init(int nx, int ny, double lx, double ly, double pi_, cudaStream_t st);
  void release();
};

// A set of device fields in the [Ny][ld] layout, allocated in one block.
template <class T>
struct FieldPool {
  Cx<T>* base = nullptr;
  size_t elems = 0;
  int count = 0;
  int alloc(const Grid<T>& g, int n, cudaStream_t st);
  Cx<T>* operator[](int i) const { return base + (size_t)i * elems; }
  void release();
};

}  // namespace tara
