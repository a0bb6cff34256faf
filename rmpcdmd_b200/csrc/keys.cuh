// Cell key of a position: cartesian_indices (src/cell_system.f90:165-175)
// followed by the compact Hilbert index, looked up in the per-box table
// built once at cell-system init.  Indices outside the table (a position
// outside the box) are hashed by the same compact-index function, which is
// what the reference does with them.
#pragma once
#include "hilbert.cuh"
#include "state.cuh"

namespace rmpcd {

__host__ __device__ inline void cell_coords(const Grid &g, double x, double y, double z, int p[3])
{
    // x / a is exact for a = 1 (every program uses a = 1): skip the division
    if (g.a != 1.0) {
        x = x / g.a;
        y = y / g.a;
        z = z / g.a;
    }
    p[0] = ifloor(x - g.origin[0]);
    p[1] = ifloor(y - g.origin[1]);
    p[2] = ifloor(z - g.origin[2]);
    if (p[0] == g.L[0]) p[0] = 0;
    if (p[1] == g.L[1]) p[1] = 0;
    if ((!g.has_walls) && (p[2] == g.L[2])) p[2] = 0;
}

__device__ inline int slot_of_cell(const Grid &g, const int p[3])
{
    if ((unsigned)p[0] < (unsigned)g.L[0] && (unsigned)p[1] < (unsigned)g.L[1] &&
        (unsigned)p[2] < (unsigned)g.L[2])
        return __ldg(g.lut + (p[0] + g.L[0] * (p[1] + g.L[1] * p[2])));
    return hilbert::compact_index(p, g.M);
}

__device__ inline int slot_of(const Grid &g, double x, double y, double z)
{
    int p[3];
    cell_coords(g, x, y, z, p);
    return slot_of_cell(g, p);
}

__device__ inline unsigned lanemask_lt()
{
    return (1u << (threadIdx.x & 31)) - 1u;
}

}  // namespace rmpcd
