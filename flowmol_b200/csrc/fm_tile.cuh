// fm_tile.cuh -- geometry of the tiled force path (single system).
//
// The extended cell grid (interior cells plus one halo layer, ne per axis) is
// cut into blocks of 2x2x2 cells.  The force kernel takes one block at a
// time: it stages the positions of every molecule a block's owners can pair
// with -- the 4x4x4 cells around the block -- in shared memory once, with the
// periodic image already applied, and evaluates each owner's list entries
// from there.  The staging order is fixed: union cell u = ux + 4 (uy + 4 uz)
// ascending (x fastest), within a cell its real members (slot ascending), then
// for a halo cell the images of the interior cell on the far side (slot
// ascending) -- two "segments" per union cell, 128 per block.  A list entry
// is the byte offset of the candidate's x in the staged tiles (16 bits).
//
// Shared-memory tiles: 32 candidates per tile, R rows of 32 doubles (x, y, z
// and, when the potential needs it, w); candidate c of the staging order sits
// at double index woff(c) = c + (c / 32) * 32 (R - 1) in row x, + 32 in row
// y, + 64 in row z, + 96 in row w (bytes: + 256, + 512, + 768).  Consecutive
// candidates are consecutive doubles of a row, so lanes that read
// neighbouring candidates hit distinct banks.  One more candidate after the
// block's capacity is a dummy far from everything (r^2 ~ 1e60, never within
// the cutoff): rows are padded with it to a whole number of loads, so the
// force loop needs no per-entry bounds test.
//
// Row layout: owner i's entries are a contiguous row of maxn16 uint16 at
// i * maxn16; with T lanes per owner, entry k sits at tile_pos16(k, T) so that
// lane l's 8-byte load of chunk c holds entries c*4T + l + T s (s = 0..3):
// the T lanes of an owner read T consecutive entries at each step.
#pragma once
#include <stdint.h>

#include "fm_common.cuh"

namespace fm {

constexpr int TILE_UE = 4;                          // union cells per axis
constexpr int TILE_NU = TILE_UE * TILE_UE * TILE_UE;  // 64 union cells
constexpr int TILE_NSEG = 2 * TILE_NU;              // real + image segment per union cell
constexpr int TILE_NSEGP = TILE_NSEG + 1;           // + the total

__host__ __device__ inline int tile_woff(int c, int R) { return c + (c >> 5) * 32 * (R - 1); }
__host__ __device__ inline int tile_boff(int c, int R) { return 8 * tile_woff(c, R); }
// candidate index of a byte offset (inverse of tile_boff on valid offsets)
__host__ __device__ inline int tile_cand(int b, int R)
{
    const int w = b >> 3;
    return (w / (32 * R)) * 32 + (w % (32 * R));
}
// Largest capacity (a multiple of 32) whose dummy candidate, index ucap, still
// has a 16-bit byte offset: R = 3: 2720, R = 4: 2016.
__host__ __device__ inline int tile_ucap_max(int R)
{
    int u = 32;
    while (tile_boff(u + 32, R) <= 65528) u += 32;
    return u;
}
// Doubles of shared memory the staging of capacity ucap (a multiple of 32)
// takes, the dummy included.
__host__ __device__ inline int tile_stage_doubles(int ucap, int R) { return (ucap / 32 + 1) * 32 * R; }

__host__ __device__ inline size_t tile_row16(int i, int maxn16) { return (size_t)i * (size_t)maxn16; }
__host__ __device__ inline int tile_pos16(int k, int T)
{
    return (k / (4 * T)) * (4 * T) + (k % T) * 4 + (k / T) % 4;
}

// Block of extended cell (cx, cy, cz) and the block's first cell.
__host__ __device__ inline int tile_block_of(const int nb[3], int cx, int cy, int cz)
{
    return (cx >> 1) + nb[0] * ((cy >> 1) + nb[1] * (cz >> 1));
}

// Segment s of the staging of the block whose first cell is (x0, y0, z0):
// the slot range [start, start + count) and the image code (NB_NOSHIFT for
// real members).  Images in a halo cell come from the interior cell on the far
// side: low halo <- last interior cell shifted by -domain, high halo <- first
// interior cell shifted by +domain (the reference's halo copy,
// messenger.serial.f90:401,509,628).
__device__ __forceinline__ void tile_segment(const int ne[3], const int32_t *cell_start, int x0, int y0, int z0,
                                             int s, int &start, int &count, int &code)
{
    const int u = s >> 1, img = s & 1;
    const int x2 = x0 - 1 + (u & 3), y2 = y0 - 1 + ((u >> 2) & 3), z2 = z0 - 1 + (u >> 4);
    start = 0;
    count = 0;
    code = 1 | (1 << 2) | (1 << 4);
    if (x2 < 0 || y2 < 0 || z2 < 0 || x2 >= ne[0] || y2 >= ne[1] || z2 >= ne[2]) return;
    if (!img) {
        const int c2 = x2 + ne[0] * (y2 + ne[1] * z2);
        start = cell_start[c2];
        count = cell_start[c2 + 1] - start;
        return;
    }
    const bool hx = x2 == 0 || x2 == ne[0] - 1, hy = y2 == 0 || y2 == ne[1] - 1, hz = z2 == 0 || z2 == ne[2] - 1;
    if (!(hx || hy || hz)) return;
    const int ssx = x2 == 0 ? -1 : (x2 == ne[0] - 1 ? 1 : 0);
    const int ssy = y2 == 0 ? -1 : (y2 == ne[1] - 1 ? 1 : 0);
    const int ssz = z2 == 0 ? -1 : (z2 == ne[2] - 1 ? 1 : 0);
    const int xs = x2 == 0 ? ne[0] - 2 : (x2 == ne[0] - 1 ? 1 : x2);
    const int ys = y2 == 0 ? ne[1] - 2 : (y2 == ne[1] - 1 ? 1 : y2);
    const int zs = z2 == 0 ? ne[2] - 2 : (z2 == ne[2] - 1 ? 1 : z2);
    const int cs2 = xs + ne[0] * (ys + ne[1] * zs);
    start = cell_start[cs2];
    count = cell_start[cs2 + 1] - start;
    code = (ssx + 1) | ((ssy + 1) << 2) | ((ssz + 1) << 4);
}

}  // namespace fm
