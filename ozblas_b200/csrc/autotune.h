// autotune.h — launch configurations chosen by measurement.
//
// Some launch choices change only speed, never bits: the order in which a
// persistent kernel's CTAs take output tiles (rasterisation strip height of
// the INT8 product, the dealing order of the grouped launch).  For those the
// first call with a new shape signature times every candidate on the real
// arguments (each candidate writes a scratch output, so the call's own output
// is written once, by the chosen configuration) and keeps the fastest.
// Choices are cached for the process and, when $OZBLAS_TUNE_CACHE names a
// file, read from and appended to it ("key choice" per line).
// $OZBLAS_TUNE=0 disables the measurement (the default candidate is used).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <functional>
#include <string>

namespace ozb {

// Returns the chosen candidate index in [0, ncand).  `run(i)` launches
// candidate i on `stream` and returns a cuozblas status; on the first use of
// `key` the default runs untimed for about 200 ms of work, then every
// candidate runs once per round, timed with CUDA events, in two rounds (the
// second in reverse order, scores summed) when the fastest time is below
// 200 ms.  When measurement is off or fails, `dflt`.
int tune_pick(const std::string &key, int ncand, int dflt, cudaStream_t stream, const std::function<int(int)> &run);

// The choice tune_pick would return without measuring: the cached candidate
// for `key`, `dflt` when measurement is off or ncand <= 1, or -1 when `key`
// has not been measured yet.
int tune_cached(const std::string &key, int ncand, int dflt);

// 64-bit FNV-1a over a byte range (shape signatures).
uint64_t tune_hash(const void *data, size_t bytes, uint64_t h = 1469598103934665603ULL);

}  // namespace ozb
