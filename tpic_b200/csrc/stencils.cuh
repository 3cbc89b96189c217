// Pointwise field stencils shared by the field kernels and their adjoints:
// the collocated N2C and C2N curls and the interior-node decoding.
#pragma once

#include "common.cuh"

namespace tpicb200 {

// NodeCellSamples::derivative, ecsim/fields/node_cell_curl.hpp:59-78: four edge
// differences summed in the written order, times 0.25 * inverse spacing.
template <class C>
__device__ __forceinline__ C edge_derivative(C d0, C d1, C d2, C d3, C inverse) {
  return C(0.25) * inverse * (d0 + d1 + d2 + d3);
}

// curl_N2C of a node field at cell (i,j,k) (node_cell_curl, :116-126).
template <class C, class T>
__device__ __forceinline__ void curl_n2c_at(const Geom& g, const T* __restrict__ f, int i, int j, int k,
                                            const C inv[3], C out[3]) {
  const long long nn = g.nodes;
  const long long b = g.node(i, j, k), sx = 1, sy = g.NX, sz = (long long)g.NX * g.NY;
  C s[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T* p = f + c * nn + b;
    // base, x, y, z, xy, xz, yz, xyz
    s[c][0] = C(p[0]); s[c][1] = C(p[sx]); s[c][2] = C(p[sy]); s[c][3] = C(p[sz]);
    s[c][4] = C(p[sx + sy]); s[c][5] = C(p[sx + sz]); s[c][6] = C(p[sy + sz]); s[c][7] = C(p[sx + sy + sz]);
  }
  // Node sources: difference = neighbor - anchor.
  auto dx = [&](const C* v) { return edge_derivative<C>(v[1] - v[0], v[5] - v[3], v[4] - v[2], v[7] - v[6], inv[0]); };
  auto dy = [&](const C* v) { return edge_derivative<C>(v[2] - v[0], v[6] - v[3], v[4] - v[1], v[7] - v[5], inv[1]); };
  auto dz = [&](const C* v) { return edge_derivative<C>(v[3] - v[0], v[5] - v[1], v[6] - v[2], v[7] - v[4], inv[2]); };
  out[0] = dy(s[2]) - dz(s[1]);
  out[1] = dz(s[0]) - dx(s[2]);
  out[2] = dx(s[1]) - dy(s[0]);
}

// curl_C2N of a cell field (with ghosts) at node (i,j,k).
template <class C, class T>
__device__ __forceinline__ void curl_c2n_at(const Geom& g, const T* __restrict__ f, int i, int j, int k,
                                            const C inv[3], C out[3]) {
  const long long nc = g.cells;
  const long long b = g.cell(i, j, k), sx = 1, sy = g.CX, sz = (long long)g.CX * g.CY;
  C s[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T* p = f + c * nc + b;
    s[c][0] = C(p[0]); s[c][1] = C(p[-sx]); s[c][2] = C(p[-sy]); s[c][3] = C(p[-sz]);
    s[c][4] = C(p[-sx - sy]); s[c][5] = C(p[-sx - sz]); s[c][6] = C(p[-sy - sz]); s[c][7] = C(p[-sx - sy - sz]);
  }
  // Cell sources: difference = anchor - neighbor.
  auto dx = [&](const C* v) { return edge_derivative<C>(v[0] - v[1], v[3] - v[5], v[2] - v[4], v[6] - v[7], inv[0]); };
  auto dy = [&](const C* v) { return edge_derivative<C>(v[0] - v[2], v[3] - v[6], v[1] - v[4], v[5] - v[7], inv[1]); };
  auto dz = [&](const C* v) { return edge_derivative<C>(v[0] - v[3], v[1] - v[5], v[2] - v[6], v[4] - v[7], inv[2]); };
  out[0] = dy(s[2]) - dz(s[1]);
  out[1] = dz(s[0]) - dx(s[2]);
  out[2] = dx(s[1]) - dy(s[0]);
}

__device__ __forceinline__ void interior_node_coordinates(const Geom& g, long long t, int& i, int& j, int& k) {
  i = int(t % g.inx);
  j = int((t / g.inx) % g.iny);
  k = int(t / ((long long)g.inx * g.iny));
}

}  // namespace tpicb200
