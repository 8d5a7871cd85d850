// Line-tile geometry shared by the generic line passes (kwb_kernels.cu, kwb_elastic.cu).
//
// A tile is 2L real lines of one axis: for x, up to 2L consecutive y rows of one z plane; for y
// and z, up to 2L consecutive x columns at one (z) or (y).  Two real lines travel as one complex
// line through the transforms.
#pragma once
#include "kwb_internal.h"

namespace kwb {

struct Tile {
  long long base;    // offset of element (column 0, position 0)
  long long stride;  // offset step along the line (strided tiles)
  int cnt;           // number of real lines (columns / rows) present in this tile
  int first_line;    // source-CSR line id of column 0
  int outer;         // z for x/y tiles, y for z tiles
  int y0;            // first row (x-direction tiles)
};

// x-direction tile: up to `rows` consecutive y rows of one z plane
__device__ __forceinline__ Tile tile_x(const SimDev &S, int rows, int tile) {
  const int Nx = S.N[0], Ny = S.N[1];
  const int tpp = (Ny + rows - 1) / rows;
  const int z = tile / tpp;
  const int y0 = (tile - z * tpp) * rows;
  Tile t;
  t.cnt = min(rows, Ny - y0);
  t.base = ((long long)z * Ny + y0) * Nx;
  t.stride = 1;
  t.first_line = y0 + Ny * z;
  t.outer = z;
  t.y0 = y0;
  return t;
}

// y- or z-direction tile of a real field: up to `cols` consecutive x columns
__device__ __forceinline__ Tile tile_yz(const SimDev &S, int axis, int cols, int tile) {
  const int Nx = S.N[0], Ny = S.N[1];
  const int tpp = (Nx + cols - 1) / cols;
  const int o = tile / tpp;
  const int x0 = (tile - o * tpp) * cols;
  Tile t;
  t.cnt = min(cols, Nx - x0);
  if (axis == 1) {
    t.base = (long long)o * Nx * Ny + x0;
    t.stride = Nx;
  } else {
    t.base = (long long)o * Nx + x0;
    t.stride = (long long)Nx * Ny;
  }
  t.first_line = x0 + Nx * o;
  t.outer = o;
  t.y0 = 0;
  return t;
}

__device__ __forceinline__ long long step_index(const SimDev &S, long long step_s) {
  return *S.t0 + step_s;
}

__device__ __forceinline__ void load_twiddles(float2 *tw, const float2 *g, int N) {
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = g[i];
}

}  // namespace kwb
