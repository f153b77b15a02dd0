// Device-wide exclusive scan, stream compaction and the 64-bit LSD radix
// sort of (Morton key, slot) pairs that orders particles each step.
//
// All three are reduce-then-scan designs: no kernel waits on another
// block, so nothing here can spin.  Work is tiled so that a block owns a
// contiguous tile and touches only its own outputs (in-place scans are safe).
#include "pot_host.h"

namespace pot {

// ---------------------------------------------------------------------------
// block-level helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= o) v += t;
	}
	return v;
}

// Exclusive block scan of one value per thread (blockDim.x = SCAN_THREADS);
// returns the exclusive prefix, writes the block total to *total.
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t* total)
{
	__shared__ uint32_t warp_tot[32];
	__shared__ uint32_t s_total;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int nw = (int)(blockDim.x >> 5);
	uint32_t inc = warp_incl_scan(v);
	if (lane == 31) warp_tot[w] = inc;
	__syncthreads();
	if (w == 0) {
		uint32_t t = (lane < nw) ? warp_tot[lane] : 0u;
		uint32_t ti = warp_incl_scan(t);
		if (lane < nw) warp_tot[lane] = ti - t;
		if (lane == 31) s_total = ti;
	}
	__syncthreads();
	const uint32_t excl = inc - v + warp_tot[w];
	*total = s_total;
	__syncthreads();  // warp_tot / s_total are reused by the next call
	return excl;
}

// ---------------------------------------------------------------------------
// scan / compaction
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ uint32_t load_val(const T* in, size_t i, size_t n)
{
	return i < n ? (uint32_t)(in[i] != 0 ? (sizeof(T) == 1 ? 1u : (uint32_t)in[i]) : 0u) : 0u;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const T* __restrict__ in, size_t n,
                                                              uint32_t* __restrict__ block_sums)
{
	const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
	uint32_t s = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) s += load_val(in, base + k, n);
	uint32_t tot;
	block_excl_scan(s, &tot);
	if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// One block scans all block sums (nb <= SCAN_TILE).
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_top(uint32_t* __restrict__ block_sums, size_t nb,
                                                           unsigned int* __restrict__ total)
{
	uint32_t v[SCAN_ITEMS];
	uint32_t s = 0;
	const size_t base = (size_t)threadIdx.x * SCAN_ITEMS;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		v[k] = (base + k < nb) ? block_sums[base + k] : 0u;
		s += v[k];
	}
	uint32_t tot;
	uint32_t run = block_excl_scan(s, &tot);
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		if (base + k < nb) block_sums[base + k] = run;
		run += v[k];
	}
	if (threadIdx.x == 0 && total) *total = tot;
}

template <typename T, bool COMPACT>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const T* __restrict__ in, size_t n,
                                                            const uint32_t* __restrict__ block_sums,
                                                            uint32_t* __restrict__ out,
                                                            uint32_t* __restrict__ prefix = nullptr)
{
	const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
	uint32_t v[SCAN_ITEMS];
	uint32_t s = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		v[k] = load_val(in, base + k, n);
		s += v[k];
	}
	uint32_t tot;
	uint32_t run = block_excl_scan(s, &tot) + block_sums[blockIdx.x];
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		if (base + k < n) {
			if (COMPACT) {
				if (v[k]) out[run] = (uint32_t)(base + k);
				if (prefix) prefix[base + k] = run;
			} else {
				out[base + k] = run;
			}
		}
		run += v[k];
		if (COMPACT && prefix && base + k + 1 == n) prefix[n] = run;
	}
}

size_t scan_blocks(size_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

void scan_exclusive(const uint32_t* in, uint32_t* out, size_t n, uint32_t* block_sums,
                    unsigned int* total, cudaStream_t s, Timer& tm)
{
	const size_t nb = scan_blocks(n ? n : 1);
	ScopedKernel k(tm, "scan", 3);
	k_scan_reduce<uint32_t><<<nb, SCAN_THREADS, 0, s>>>(in, n, block_sums);
	k_scan_top<<<1, SCAN_THREADS, 0, s>>>(block_sums, nb, total);
	k_scan_down<uint32_t, false><<<nb, SCAN_THREADS, 0, s>>>(in, n, block_sums, out);
}

void compact_flags(const uint8_t* flags, size_t n, uint32_t* list, uint32_t* block_sums,
                   unsigned int* count, cudaStream_t s, Timer& tm, uint32_t* prefix)
{
	const size_t nb = scan_blocks(n ? n : 1);
	ScopedKernel k(tm, "compact", 3);
	k_scan_reduce<uint8_t><<<nb, SCAN_THREADS, 0, s>>>(flags, n, block_sums);
	k_scan_top<<<1, SCAN_THREADS, 0, s>>>(block_sums, nb, count);
	k_scan_down<uint8_t, true><<<nb, SCAN_THREADS, 0, s>>>(flags, n, block_sums, list, prefix);
}

// ---------------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------------
// Per-tile digit histogram, written digit-major: counts[d * nb + b].
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint64_t* __restrict__ keys, size_t n, int shift,
                                                        uint32_t* __restrict__ counts, uint32_t nb)
{
	__shared__ uint32_t h[8][RS_BINS];
	const int w = threadIdx.x >> 5;
	for (int i = threadIdx.x; i < 8 * RS_BINS; i += RS_THREADS) (&h[0][0])[i] = 0;
	__syncthreads();
	const size_t base = (size_t)blockIdx.x * RS_TILE + threadIdx.x;
#pragma unroll 4
	for (int r = 0; r < RS_ITEMS; r++) {
		const size_t i = base + (size_t)r * RS_THREADS;
		if (i < n) atomicAdd(&h[w][(keys[i] >> shift) & 0xFF], 1u);
	}
	__syncthreads();
	const int d = threadIdx.x;  // RS_THREADS == RS_BINS
	uint32_t c = 0;
#pragma unroll
	for (int k = 0; k < 8; k++) c += h[k][d];
	counts[(size_t)d * nb + blockIdx.x] = c;
}

// Stable scatter: tile processed in RS_ITEMS rounds of RS_THREADS keys in
// index order; within a round the rank of a key among equal digits is
// (earlier rounds) + (earlier warps this round) + (earlier lanes).
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint64_t* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin, size_t n,
                                                           int shift, const uint32_t* __restrict__ offsets,
                                                           uint32_t nb, uint64_t* __restrict__ kout,
                                                           uint32_t* __restrict__ vout)
{
	__shared__ uint32_t s_base[RS_BINS];
	__shared__ uint32_t s_tot[RS_BINS];
	__shared__ uint32_t s_wcnt[8][RS_BINS];
	__shared__ uint32_t s_wpre[8][RS_BINS];
	const int t = threadIdx.x, w = t >> 5, lane = t & 31;
	const uint32_t lt_mask = (1u << lane) - 1u;
	s_base[t] = offsets[(size_t)t * nb + blockIdx.x];
#pragma unroll
	for (int k = 0; k < 8; k++) s_wcnt[k][t] = 0;
	__syncthreads();
	const size_t base = (size_t)blockIdx.x * RS_TILE;
	for (int r = 0; r < RS_ITEMS; r++) {
		const size_t i = base + (size_t)r * RS_THREADS + t;
		const bool valid = i < n;
		uint64_t key = 0;
		uint32_t val = 0;
		int d = RS_BINS;  // sentinel for the ragged tail
		if (valid) {
			key = kin[i];
			val = vin[i];
			d = (int)((key >> shift) & 0xFF);
		}
		const uint32_t peers = __match_any_sync(0xffffffffu, d);
		const uint32_t lrank = __popc(peers & lt_mask);
		if (valid && lrank == 0) s_wcnt[w][d] = __popc(peers);
		__syncthreads();
		{
			uint32_t run = 0;
#pragma unroll
			for (int k = 0; k < 8; k++) {
				const uint32_t c = s_wcnt[k][t];
				s_wcnt[k][t] = 0;
				s_wpre[k][t] = run;
				run += c;
			}
			s_tot[t] = run;
		}
		__syncthreads();
		if (valid) {
			const uint32_t pos = s_base[d] + s_wpre[w][d] + lrank;
			kout[pos] = key;
			vout[pos] = val;
		}
		__syncthreads();
		s_base[t] += s_tot[t];
	}
}

size_t radix_counts_words(size_t n)
{
	const size_t nb = (n + RS_TILE - 1) / RS_TILE;
	return (size_t)RS_BINS * (nb ? nb : 1);
}

void radix_sort_pairs(uint64_t* keys[2], uint32_t* vals[2], size_t n, uint32_t* counts,
                      uint32_t* block_sums, cudaStream_t s, Timer& tm)
{
	if (n == 0) return;
	const uint32_t nb = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
	const size_t nc = (size_t)RS_BINS * nb;
	int src = 0;
	for (int pass = 0; pass < 8; pass++) {
		const int shift = 8 * pass;
		{
			ScopedKernel k(tm, "sort_hist");
			k_rs_hist<<<nb, RS_THREADS, 0, s>>>(keys[src], n, shift, counts, nb);
		}
		scan_exclusive(counts, counts, nc, block_sums, nullptr, s, tm);
		{
			ScopedKernel k(tm, "sort_scatter");
			k_rs_scatter<<<nb, RS_THREADS, 0, s>>>(keys[src], vals[src], n, shift, counts, nb,
			                                       keys[src ^ 1], vals[src ^ 1]);
		}
		src ^= 1;
	}
}

}  // namespace pot
