// Device-wide exclusive scan, stream compaction and the 64-bit LSD radix
// sort of (Morton key, slot) pairs that orders particles each step.
//
// The scan and the compaction are reduce-then-scan designs: none of their
// kernels waits on another block.  The radix sort's pass (k_os_pass) does
// wait: each tile spins in its decoupled look-back on the status words of
// tiles that took an earlier ticket (and are therefore resident), with
// OS_SPIN_CAP as the limit after which it records POT_E_ITER and finishes.
// Work is tiled so that a block owns a contiguous tile and touches only its
// own outputs (in-place scans are safe).
#include "pot_tree.cuh"

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

template <typename T, class G>
__device__ __forceinline__ void scan_reduce_body(G grd, const T* __restrict__ in, size_t n,
                                                 uint32_t* __restrict__ block_sums)
{
	const size_t base = (size_t)grd.id() * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
	uint32_t s = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) s += load_val(in, base + k, n);
	uint32_t tot;
	block_excl_scan(s, &tot);
	if (threadIdx.x == 0) block_sums[grd.id()] = tot;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const T* __restrict__ in, size_t n,
                                                              uint32_t* __restrict__ block_sums)
{
	scan_reduce_body<T>(GridSelf {}, in, n, block_sums);
}

// One block scans all block sums (nb <= SCAN_TILE).
template <class G>
__device__ __forceinline__ void scan_top_body(G grd, uint32_t* __restrict__ block_sums, size_t nb,
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

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_top(uint32_t* __restrict__ block_sums, size_t nb,
                                                           unsigned int* __restrict__ total)
{
	scan_top_body(GridSelf {}, block_sums, nb, total);
}

template <typename T, bool COMPACT, class G>
__device__ __forceinline__ void scan_down_body(G grd, const T* __restrict__ in, size_t n,
                                               const uint32_t* __restrict__ block_sums, uint32_t* __restrict__ out,
                                               uint32_t* __restrict__ prefix)
{
	const size_t base = (size_t)grd.id() * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
	uint32_t v[SCAN_ITEMS];
	uint32_t s = 0;
#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		v[k] = load_val(in, base + k, n);
		s += v[k];
	}
	uint32_t tot;
	uint32_t run = block_excl_scan(s, &tot) + block_sums[grd.id()];
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

template <typename T, bool COMPACT>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const T* __restrict__ in, size_t n,
                                                            const uint32_t* __restrict__ block_sums,
                                                            uint32_t* __restrict__ out,
                                                            uint32_t* __restrict__ prefix = nullptr)
{
	scan_down_body<T, COMPACT>(GridSelf {}, in, n, block_sums, out, prefix);
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
                   unsigned int* count, cudaStream_t s, Timer& tm, uint32_t* prefix, bool tiles_counted)
{
	const size_t nb = scan_blocks(n ? n : 1);
	ScopedKernel k(tm, "compact", tiles_counted ? 2 : 3);
	if (!tiles_counted) k_scan_reduce<uint8_t><<<nb, SCAN_THREADS, 0, s>>>(flags, n, block_sums);
	k_scan_top<<<1, SCAN_THREADS, 0, s>>>(block_sums, nb, count);
	k_scan_down<uint8_t, true><<<nb, SCAN_THREADS, 0, s>>>(flags, n, block_sums, list, prefix);
}

// ---------------------------------------------------------------------------
// radix sort: one kernel per 8-bit pass with decoupled look-back
// ---------------------------------------------------------------------------
// Tiles of OS_TILE keys.  The grid is the blocks the device holds at once;
// each block takes the next tile index from a counter (so tiles start in
// index order) until none is left, ranks its keys stably per digit, publishes
// its per-digit counts, and obtains the exclusive prefix of each digit over
// all earlier tiles by looking back at their published words (aggregate or
// inclusive prefix).  Every wait has an iteration cap; reaching it records
// POT_E_ITER and the pass completes with wrong order but without hanging.
// The keys are then staged in shared memory in digit order and written out
// contiguously per digit.
constexpr int OS_THREADS = 256;
constexpr int OS_ITEMS = 8;
constexpr int OS_TILE = OS_THREADS * OS_ITEMS;
constexpr uint32_t OS_FLAG_AGG = 1u << 30;
constexpr uint32_t OS_FLAG_PRE = 2u << 30;
constexpr uint32_t OS_COUNT = (1u << 30) - 1u;
constexpr long OS_SPIN_CAP = 1L << 24;
constexpr int OS_LOOKBACK = 8;      // earlier tiles read per round of the look-back

// In place: hist[p * 256 + d] <- exclusive prefix over digits (one block).
template <class G>
__device__ __forceinline__ void os_offsets_body(G grd, uint32_t* __restrict__ hist, int npass)
{
	for (int p = 0; p < npass; p++) {
		uint32_t tot;
		const uint32_t v = hist[p * RS_BINS + threadIdx.x];
		const uint32_t e = block_excl_scan(v, &tot);
		hist[p * RS_BINS + threadIdx.x] = e;
		__syncthreads();
	}
}

__global__ void __launch_bounds__(RS_BINS) k_os_offsets(uint32_t* __restrict__ hist, int npass)
{
	os_offsets_body(GridSelf {}, hist, npass);
}

template <class G>
__device__ __forceinline__ void os_pass_body(G grd, const uint64_t* __restrict__ kin,
                                             const uint32_t* __restrict__ vin, size_t n, int shift,
                                             const uint32_t* __restrict__ goff, uint32_t* __restrict__ status,
                                             unsigned int* __restrict__ tile_ctr, uint64_t* __restrict__ kout,
                                             uint32_t* __restrict__ vout, int* __restrict__ err)
{
	constexpr int NW = OS_THREADS / 32;
	__shared__ uint32_t s_tile;
	__shared__ uint32_t s_wcnt[NW][RS_BINS];  // per-warp running count, then per-warp exclusive prefix
	__shared__ uint32_t s_loc[RS_BINS];       // digit start inside the staged tile
	__shared__ uint32_t s_glob[RS_BINS];      // digit start in the output
	__shared__ uint64_t s_key[OS_TILE];
	__shared__ uint32_t s_val[OS_TILE];
	const int t = threadIdx.x, w = t >> 5, lane = t & 31;
	const uint32_t lt_mask = (1u << lane) - 1u;
	for (;;) {  // tiles in ticket order until none is left
		if (t == 0) s_tile = atomicAdd(tile_ctr, 1u);
#pragma unroll
		for (int k = 0; k < NW; k++) s_wcnt[k][t] = 0;
		__syncthreads();
		const uint32_t tile = s_tile;
		const size_t base = (size_t)tile * OS_TILE;
		if (base >= n) return;
		// warp w holds the tile's keys [256 w, 256 w + 256), round r the 32 at
		// 256 w + 32 r, so a key's index in the tile is (warp, round, lane) in order
		uint64_t key[OS_ITEMS];
		uint32_t val[OS_ITEMS];
		uint32_t rank[OS_ITEMS];
		int dig[OS_ITEMS];
#pragma unroll
		for (int r = 0; r < OS_ITEMS; r++) {
			const size_t i = base + (size_t)(w * 32 * OS_ITEMS + r * 32 + lane);
			dig[r] = RS_BINS;
			key[r] = 0;
			val[r] = 0;
			if (i < n) {
				key[r] = kin[i];
				val[r] = vin[i];
				dig[r] = (int)((key[r] >> shift) & 0xFF);
			}
		}
		// stable ranks inside the warp: a running count per digit in the warp's
		// own row, updated once per round by the lowest lane of each digit
#pragma unroll
		for (int r = 0; r < OS_ITEMS; r++) {
			const int d = dig[r];
			const uint32_t peers = __match_any_sync(0xffffffffu, d);
			const uint32_t before = d < RS_BINS ? s_wcnt[w][d] : 0u;
			rank[r] = before + __popc(peers & lt_mask);
			__syncwarp();
			if (d < RS_BINS && (peers & lt_mask) == 0u) s_wcnt[w][d] = before + __popc(peers);
			__syncwarp();
		}
		__syncthreads();
		// digit t: each warp's exclusive prefix over the warps before it, and
		// the tile's count
		uint32_t cnt = 0;
#pragma unroll
		for (int k = 0; k < NW; k++) {
			const uint32_t c = s_wcnt[k][t];
			s_wcnt[k][t] = cnt;
			cnt += c;
		}
		// publish this tile's count of digit t, then look back for its prefix,
		// OS_LOOKBACK earlier tiles per round of reads
		volatile uint32_t* st = status;
		st[(size_t)tile * RS_BINS + t] = (tile == 0 ? OS_FLAG_PRE : OS_FLAG_AGG) | cnt;
		uint32_t excl = 0;
		if (tile > 0) {
			long spins = 0;
			int64_t j = (int64_t)tile - 1;  // next tile to read
			bool found = false;
			while (!found) {
				uint32_t v[OS_LOOKBACK];
#pragma unroll
				for (int q = 0; q < OS_LOOKBACK; q++) v[q] = j - q >= 0 ? st[(size_t)(j - q) * RS_BINS + t] : 0u;
				int used = 0;
				bool stalled = false;
#pragma unroll
				for (int q = 0; q < OS_LOOKBACK; q++) {
					if (found || stalled) continue;
					const uint32_t flag = v[q] & ~OS_COUNT;
					if (flag == 0) {  // not yet published (tile 0 always is, so j - q >= 0 here)
						stalled = true;
						continue;
					}
					excl += v[q] & OS_COUNT;
					used++;
					if (flag == OS_FLAG_PRE) found = true;
				}
				if (found) break;
				j -= used;
				if (used == 0 && ++spins > OS_SPIN_CAP) {
					atomicCAS(err, 0, POT_E_ITER);
					break;
				}
			}
			st[(size_t)tile * RS_BINS + t] = OS_FLAG_PRE | (excl + cnt);
		}
		s_glob[t] = goff[t] + excl;
		// digit starts inside the tile
		{
			uint32_t tot;
			const uint32_t e = block_excl_scan(cnt, &tot);
			s_loc[t] = e;
		}
		__syncthreads();
#pragma unroll
		for (int r = 0; r < OS_ITEMS; r++) {
			if (dig[r] < RS_BINS) {
				const uint32_t p = s_loc[dig[r]] + s_wcnt[w][dig[r]] + rank[r];
				s_key[p] = key[r];
				s_val[p] = val[r];
			}
		}
		__syncthreads();
		const uint32_t nt = (uint32_t)((n - base) < (size_t)OS_TILE ? (n - base) : (size_t)OS_TILE);
		for (uint32_t i = t; i < nt; i += OS_THREADS) {
			const uint64_t k = s_key[i];
			const int d = (int)((k >> shift) & 0xFF);
			const uint32_t o = s_glob[d] + (i - s_loc[d]);
			kout[o] = k;
			vout[o] = s_val[i];
		}
		__syncthreads();  // the next tile reuses the shared arrays
	}
}

__global__ void __launch_bounds__(OS_THREADS) k_os_pass(const uint64_t* __restrict__ kin,
                                                        const uint32_t* __restrict__ vin, size_t n, int shift,
                                                        const uint32_t* __restrict__ goff,
                                                        uint32_t* __restrict__ status,
                                                        unsigned int* __restrict__ tile_ctr,
                                                        uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                        int* __restrict__ err)
{
	os_pass_body(GridSelf {}, kin, vin, n, shift, goff, status, tile_ctr, kout, vout, err);
}

static inline int os_passes(int low_bit) { return (63 - low_bit + 7) / 8; }

// Blocks of k_os_pass resident on the device at once: the pass's grid, each
// block taking tiles until none is left (no second wave of blocks).
static uint32_t os_resident()
{
	static uint32_t n = 0;
	if (!n) {
		int dev = 0, sms = 0, per = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_os_pass, OS_THREADS, 0);
		n = (uint32_t)std::max(1, sms) * (uint32_t)std::max(1, per);
	}
	return n;
}

uint32_t radix_tiles(size_t n) { return (uint32_t)((n + OS_TILE - 1) / OS_TILE); }
int radix_passes(int low_bit) { return os_passes(low_bit); }

size_t radix_counts_words(size_t n)
{
	const size_t tiles = (n + OS_TILE - 1) / OS_TILE;
	return (size_t)OS_MAX_PASSES * (tiles ? tiles : 1) * RS_BINS + (size_t)OS_MAX_PASSES * RS_BINS + OS_MAX_PASSES;
}

uint32_t* radix_sort_begin(uint32_t* counts, size_t n, int low_bit, cudaStream_t s)
{
	const uint32_t tiles = (uint32_t)((n + OS_TILE - 1) / OS_TILE);
	const int npass = os_passes(low_bit);
	uint32_t* hist = counts + (size_t)OS_MAX_PASSES * tiles * RS_BINS;
	cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)npass * tiles * RS_BINS, s);
	cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (OS_MAX_PASSES * RS_BINS + OS_MAX_PASSES), s);
	return hist;
}

int radix_sort_pairs(uint64_t* keys[2], uint32_t* vals[2], size_t n, uint32_t* counts, uint32_t* block_sums,
                     int low_bit, cudaStream_t s, Timer& tm, int* err)
{
	(void)block_sums;
	if (n == 0) return 0;
	const uint32_t tiles = (uint32_t)((n + OS_TILE - 1) / OS_TILE);
	const int npass = os_passes(low_bit);
	uint32_t* status = counts;
	uint32_t* hist = counts + (size_t)OS_MAX_PASSES * tiles * RS_BINS;
	unsigned int* ctr = hist + OS_MAX_PASSES * RS_BINS;
	{
		ScopedKernel k(tm, "sort_offsets");
		k_os_offsets<<<1, RS_BINS, 0, s>>>(hist, npass);
	}
	int src = 0;
	for (int p = 0; p < npass; p++) {
		ScopedKernel k(tm, "sort_pass");
		const uint32_t grid = std::min<uint32_t>(tiles, os_resident());
		k_os_pass<<<grid, OS_THREADS, 0, s>>>(keys[src], vals[src], n, low_bit + 8 * p, hist + p * RS_BINS,
		                                      status + (size_t)p * tiles * RS_BINS, ctr + p, keys[src ^ 1],
		                                      vals[src ^ 1], err);
		src ^= 1;
	}
	return src;
}

}  // namespace pot

// ---------------------------------------------------------------------------
// packed batch: the sort, the due list and the cell numbering of every
// member in one launch per kernel (the single run's sequences above)
// ---------------------------------------------------------------------------
namespace pot {

uint32_t pack_scan_blocks(uint32_t n) { return (uint32_t)scan_blocks(n ? n : 1); }

// scan_blocks(max(n, 1)) in device code
__device__ __forceinline__ size_t dev_scan_blocks(size_t n)
{
	return ((n ? n : 1) + SCAN_TILE - 1) / SCAN_TILE;
}

// The radix sort's layout in a member's counts buffer (radix_sort_pairs).
struct OsLayout {
	uint32_t* status;
	uint32_t* hist;
	unsigned int* ctr;
	__device__ OsLayout(const MemberView& v)
	{
		status = v.counts;
		hist = v.counts + (size_t)OS_MAX_PASSES * v.tiles * RS_BINS;
		ctr = hist + OS_MAX_PASSES * RS_BINS;
	}
};

// What the single run clears with memsets before its sort, tree and groups:
// each tile's status words of every pass; block 0 of a member the digit
// counts, tile counters, due-flag tile counts, overflow count and group count.
__global__ void __launch_bounds__(OS_THREADS) kp_sort_clear(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_TILES], B.M);
	const MemberView& v = B.mv[sb.m];
	const OsLayout L(v);
	for (uint32_t p = 0; p < B.npass; p++)
		L.status[((size_t)p * v.tiles + sb.id) * RS_BINS + threadIdx.x] = 0u;
	if (sb.id == 0) {
		for (int i = threadIdx.x; i < OS_MAX_PASSES * RS_BINS + OS_MAX_PASSES; i += OS_THREADS) L.hist[i] = 0u;
		const uint32_t nt = (uint32_t)dev_scan_blocks(v.P.n);
		for (uint32_t i = threadIdx.x; i < nt; i += OS_THREADS) v.due_tiles[i] = 0u;
		if (threadIdx.x == 0) {
			v.rec->n_overflow = 0;
			v.rec->n_groups = 0;
		}
	}
}

__global__ void __launch_bounds__(RS_BINS) kp_os_offsets(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_ONE], B.M);
	const MemberView& v = B.mv[sb.m];
	os_offsets_body(GridSeg { sb.id, sb.n }, OsLayout(v).hist, (int)B.npass);
}

// Pass p: every member's tiles; a tile's index within its member comes from
// the member's own ticket counter, so the look-back waits only on tiles of
// the same member that took earlier tickets (and are therefore resident).
__global__ void __launch_bounds__(OS_THREADS) kp_os_pass(PackDev B, int p)
{
	const SegBlock sb = seg_block(B.pre[PS_TILES], B.M);
	const MemberView& v = B.mv[sb.m];
	const OsLayout L(v);
	const int src = p & 1;
	os_pass_body(GridSeg { sb.id, sb.n }, v.keys[src], v.vals[src], (size_t)v.P.n, (int)v.P.key_bits + 8 * p,
	             L.hist + p * RS_BINS, L.status + (size_t)p * v.tiles * RS_BINS, L.ctr + p, v.keys[src ^ 1],
	             v.vals[src ^ 1], &v.rec->status);
}

void pack_sort_begin(const PackDev& B, cudaStream_t s)
{
	kp_sort_clear<<<B.blocks[PS_TILES], OS_THREADS, 0, s>>>(B);
}

void pack_sort(const PackDev& B, cudaStream_t s)
{
	kp_os_offsets<<<B.blocks[PS_ONE], RS_BINS, 0, s>>>(B);
	for (uint32_t p = 0; p < B.npass; p++) kp_os_pass<<<B.blocks[PS_TILES], OS_THREADS, 0, s>>>(B, (int)p);
}

// the due list and its prefix (compact_flags; the reorder counted each tile)
__global__ void __launch_bounds__(SCAN_THREADS) kp_cmp_top(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_ONE], B.M);
	const MemberView& v = B.mv[sb.m];
	scan_top_body(GridSeg { sb.id, sb.n }, v.due_tiles, dev_scan_blocks(v.P.n), &v.rec->n_due);
}

__global__ void __launch_bounds__(SCAN_THREADS) kp_cmp_down(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_CMP], B.M);
	const MemberView& v = B.mv[sb.m];
	scan_down_body<uint8_t, true>(GridSeg { sb.id, sb.n }, v.due, (size_t)v.P.n, v.due_tiles, v.due_list,
	                              v.due_prefix);
}

void pack_compact(const PackDev& B, cudaStream_t s)
{
	kp_cmp_top<<<B.blocks[PS_ONE], SCAN_THREADS, 0, s>>>(B);
	kp_cmp_down<<<B.blocks[PS_CMP], SCAN_THREADS, 0, s>>>(B);
}

// cell numbering: exclusive scan of the cells each key pair owns
// (launch_build's scan_exclusive)
__global__ void __launch_bounds__(SCAN_THREADS) kp_node_reduce(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_NODES], B.M);
	const MemberView& v = B.mv[sb.m];
	scan_reduce_body<uint32_t>(GridSeg { sb.id, sb.n }, v.T.cnt, (size_t)(v.P.n_tree - v.P.leaf_size),
	                           v.block_sums);
}

__global__ void __launch_bounds__(SCAN_THREADS) kp_node_top(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_ONE], B.M);
	const MemberView& v = B.mv[sb.m];
	const size_t np = v.P.n_tree - v.P.leaf_size;
	scan_top_body(GridSeg { sb.id, sb.n }, v.block_sums, dev_scan_blocks(np), &v.rec->n_nodes);
}

__global__ void __launch_bounds__(SCAN_THREADS) kp_node_down(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_NODES], B.M);
	const MemberView& v = B.mv[sb.m];
	scan_down_body<uint32_t, false>(GridSeg { sb.id, sb.n }, v.T.cnt, (size_t)(v.P.n_tree - v.P.leaf_size),
	                                v.block_sums, v.T.base, nullptr);
}

void pack_node_scan(const PackDev& B, cudaStream_t s)
{
	kp_node_reduce<<<B.blocks[PS_NODES], SCAN_THREADS, 0, s>>>(B);
	kp_node_top<<<B.blocks[PS_ONE], SCAN_THREADS, 0, s>>>(B);
	kp_node_down<<<B.blocks[PS_NODES], SCAN_THREADS, 0, s>>>(B);
}

}  // namespace pot
