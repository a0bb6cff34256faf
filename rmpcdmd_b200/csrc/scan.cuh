// Exclusive prefix sum over the Hilbert-slot counts (the serial prefix of
// src/cell_system.f90:124-127): three launches -- per-block totals, a scan of
// the block totals in one block, and the block-offset rescan that writes the
// starts (and, optionally, a second copy used as scatter cursors).
#pragma once
#include "rmpcd_common.cuh"

namespace rmpcd {

constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 4;
constexpr int kScanTile = kScanThreads * kScanPerThread;

inline int scan_blocks_for(int n) { return (n + kScanTile - 1) / kScanTile; }

// Launches the three-phase scan.  block_tmp must hold scan_blocks_for(n)
// ints; n_blocks <= 16 * kScanThreads.  If zero_in is set, the input array is
// cleared after it has been read (so it can accumulate the next counts).
int exclusive_scan(int *in, int *out, int *out2, int n, int *block_tmp, bool zero_in,
                   cudaStream_t s);

}  // namespace rmpcd
