// Host-side launch wrappers shared by the kernel translation units, and the
// per-kernel event timer used when POT_OPT_TIMING is set.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "pot_internal.cuh"

namespace pot {

// Records a start/stop event pair around each kernel when enabled; the
// pairs are resolved into per-name totals at the next sync point.
class Timer {
public:
	bool enabled = false;
	cudaStream_t stream = nullptr;
	uint64_t launches = 0;  // kernels enqueued through ScopedKernel scopes (always counted)

	void begin(const char* name);
	void end();
	void resolve();   // stream must be idle
	void reset();
	int report(int max, const char** names, double* ms, uint64_t* launches) const;
	~Timer();

private:
	struct Pending { int kind; cudaEvent_t a, b; };
	std::vector<const char*> names_;
	std::vector<double> ms_;
	std::vector<uint64_t> count_;
	std::vector<Pending> pending_;
	std::vector<cudaEvent_t> pool_;
	int open_kind_ = -1;
	cudaEvent_t open_a_ = nullptr;
	cudaEvent_t take();
	int kind_of(const char* name);
};

struct ScopedKernel {
	Timer& t;
	ScopedKernel(Timer& tm, const char* name, int kernels = 1) : t(tm)
	{
		t.launches += (uint64_t)kernels;
		t.begin(name);
	}
	~ScopedKernel() { t.end(); }
};

// ---- sort.cu ------------------------------------------------------------
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_BINS = 256;
constexpr int OS_MAX_PASSES = 8;  // radix passes at most (64-bit keys, 8 bits each)

size_t scan_blocks(size_t n);
// out[i] = sum in[0..i); *total = sum of all (device pointer, may be null).
void scan_exclusive(const uint32_t* in, uint32_t* out, size_t n, uint32_t* block_sums,
                    unsigned int* total, cudaStream_t s, Timer& tm);
// list[k] = i for the k-th i with flags[i] != 0; *count = number of such i;
// prefix (optional, n + 1 entries) = exclusive prefix sum of the flags.
// tiles_counted: block_sums already holds each scan tile's count of set
// flags (the producer counted them), so the first stage is skipped.
void compact_flags(const uint8_t* flags, size_t n, uint32_t* list, uint32_t* block_sums,
                   unsigned int* count, cudaStream_t s, Timer& tm, uint32_t* prefix = nullptr,
                   bool tiles_counted = false);
size_t radix_counts_words(size_t n);
// LSD radix sort of (keys, vals) on bits [low_bit, 64) in 8-bit passes;
// result in keys[0]/vals[0] when the number of passes is even, keys[1]/vals[1]
// otherwise (returns the index).
// tiles and 8-bit passes of radix_sort_pairs for n keys sorted from low_bit
uint32_t radix_tiles(size_t n);
int radix_passes(int low_bit);
// Clear the sort's status words, digit counts and tile counters before the
// keys are written; returns the digit-count array (OS_MAX_PASSES x 256) that
// the keys kernel fills as it writes the keys.
uint32_t* radix_sort_begin(uint32_t* counts, size_t n, int low_bit, cudaStream_t s);
// After radix_sort_begin and the keys kernel's digit counts:
int radix_sort_pairs(uint64_t* keys[2], uint32_t* vals[2], size_t n, uint32_t* counts, uint32_t* block_sums,
                     int low_bit, cudaStream_t s, Timer& tm, int* err);

}  // namespace pot
