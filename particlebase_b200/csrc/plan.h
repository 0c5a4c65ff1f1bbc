// Host-side planning shared by the single-system and batched paths:
// the reference cell grid, Morton ranking of (x, y) columns and the force
// work items.
#pragma once

#include <cstdint>
#include <vector>

#include "md.cuh"

namespace pb {

// cudaCutoffBlock::setupCutoffBlock (cudaCutoffBlock.cu:97-113) in the same
// FP32 operations.  Periodic: blocknum = (uint32)(c / rmax),
// blocklen = c / (float)blocknum.  Open boundaries: blocklen = rmax and
// blocknum = (uint32)(c / rmax) + 1, one block past the top face.  Returns
// false if any axis has < 3 cells (the reference asserts blocknum > 2).
bool make_grid(const float cell6[6], float rmax, Grid &g, bool periodic = true);

// rank[d0 * ny + d1] = position of column (d0, d1) along a Z-order curve;
// xy[rank] = d0 * ny + d1.
void morton_columns(int nx, int ny, std::vector<uint32_t> &rank, std::vector<uint32_t> &xy);

// Reference 27-neighbour table (calc_BlockNeighbor, cudaCutoffBlock.cu:17-65)
// in reference cell numbering d2 + d1 nz + d0 nz ny; in an open box a
// neighbour outside the grid is kNoCell.
void neighbor_table(const Grid &g, std::vector<uint32_t> &out);

// z cells per force work item for a mean cell occupancy: about 200 * scale
// home atoms per item, at most force_max_segment(), and short enough for two
// force CTAs per SM with `nt` atom types.
// `half`: the half-shell force kernel runs (its stage has to fit as well).
int choose_segment(double atoms_per_cell, int nz, double scale = 1.0, int nt = 1,
                   bool half = false);

// Shared-memory capacity (atoms) of a force CTA staging 9 columns x (seg + 2)
// cells at the given mean occupancy, with headroom for fluctuations.
int choose_capacity(double atoms_per_cell, int seg);
// Member slots per cell bucket of the two-kernel cell build: at least 32 and
// about twice the mean occupancy (a fuller cell spills to the overflow list).
int choose_bucket_cap(double atoms_per_cell);
// Members a 64-cell tile block of the cell build stages in shared memory
// (9 B each): about 1.3 times the mean tile; fuller tiles take the slower path.
int choose_tile_atoms(double atoms_per_cell);
// The same for the half-shell force kernel, which stages 5 columns.
int choose_capacity_half(double atoms_per_cell, int seg);

// Force work items of one system whose packed cell keys start at cell0, with
// the column ranking `rank` (reference column -> rank) and its inverse `xy`.
void append_items(uint32_t sys, const Grid &g, int seg, uint32_t cell0,
                  const std::vector<uint32_t> &rank, const std::vector<uint32_t> &xy,
                  std::vector<ForceItem> &items);

int force_max_segment();
// Largest staged-atom capacity of a force CTA of `warps` warps for `nt` types.
int force_max_capacity(int warps, int nt);
// Shared memory (dynamic plus an upper bound of the static part) of one
// default-shape force CTA with staged-atom capacity `cap` and `nt` types.
int force_smem_per_cta(int cap, int nt);
// The shared memory a default-shape force CTA may use so that the CTAs per SM
// its launch shape is built for stay resident.
int force_smem_limit();
// The same two for the half-shell force kernel (force_half.cu).
int force_half_max_capacity(int nt);
int force_half_smem_per_cta(int cap, int nt);

}  // namespace pb
