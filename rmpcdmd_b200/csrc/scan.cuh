// Exclusive prefix sum over the Hilbert-slot counts (the serial prefix of
// src/cell_system.f90:124-127) in two launches: the total of every tile of
// kScanTile slots, then one block per tile that adds the totals of the tiles
// before it and scans its own tile.
#pragma once
#include "rmpcd_common.cuh"

namespace rmpcd {

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;
constexpr int kScanTile = kScanThreads * kScanPerThread;
// a block reads the totals of up to kScanMaxTiles - 1 earlier tiles (128
// loads per thread at the maximum, 2^27 slots: the largest cell system)
constexpr int kScanMaxTiles = 128 * kScanThreads;

inline int scan_blocks_for(int n) { return (n + kScanTile - 1) / kScanTile; }

// Writes the exclusive scan of in[0..n) to out (and out2 when not null) and,
// when clear is not null, zeroes clear[0..n) (an array distinct from in that
// accumulates the next counts).  tile_total holds scan_blocks_for(n) ints;
// in, out, out2 and clear are 16-byte aligned.
int exclusive_scan(const int *in, int *out, int *out2, int n, int *tile_total, int *clear, cudaStream_t s);

}  // namespace rmpcd
