// Morton keys, per-step reorder, octree build and upward moments.
//
// Topology.  The reference inserts particles one by one into a pointer
// octree whose root is [0, 2 r mpp]^3 and whose cells split at the midpoint
// (x1 + x2) / 2 of their faces until every leaf holds one particle
// (pot.c:1457-1643).  The final tree does not depend on insertion order: a
// cell is internal exactly when two or more particles lie in it.  So it is
// rebuilt here from sorted keys:
//   * key = 21 levels x 3 bits of the comparisons `x < mid` the reference's
//     descent makes (pot.c:1522-1553), computed with the same midpoint
//     arithmetic, so cell membership is bit-identical;
//   * with keys sorted, the cell of level l containing particle i holds
//     more than L particles iff keys i and i + L share its 3l-bit prefix;
//     pair i = (i, i + L) "owns" the cells whose first particle is i, i.e.
//     the levels (lvl[i-1], lvl[i]], which numbers cells in pre-order;
//   * a cell's last particle and its 8 children are found by searches over
//     its key range that make several independent reads per round
//     (cell_end, child_starts).
// Leaf size L = 1 reproduces the reference's tree; L > 1 gives bucket leaves.
//
// Moments.  Net charge q, absolute charge aq and the |q|-weighted centre of
// a cell are the reference's running update over its children in the
// member order gxlylz, gxlygz, lxlylz, lxlygz, lxgylz, lxgygz, gxgylz, gxgygz
// (pot.c:1290-1402), evaluated bottom-up with arrival counters and unfused
// double operations, which makes them bit-identical too.
#include "pot_tree.cuh"

namespace pot {

// 63-bit key: level 1 in bits 62..60, digit = gx << 2 | gy << 1 | gz.
__device__ __forceinline__ uint64_t morton_key(double x, double y, double z, double w)
{
	double lx = 0.0, hx = w, ly = 0.0, hy = w, lz = 0.0, hz = w;
	uint64_t key = 0;
#pragma unroll 3
	for (int l = 0; l < MAX_LEVELS; l++) {
		const double mx = dmul(dadd(lx, hx), 0.5);
		const double my = dmul(dadd(ly, hy), 0.5);
		const double mz = dmul(dadd(lz, hz), 0.5);
		const uint32_t bx = (x < mx) ? 0u : 1u;
		const uint32_t by = (y < my) ? 0u : 1u;
		const uint32_t bz = (z < mz) ? 0u : 1u;
		if (bx) lx = mx; else hx = mx;
		if (by) ly = my; else hy = my;
		if (bz) lz = mz; else hz = mz;
		key = (key << 3) | (uint64_t)((bx << 2) | (by << 1) | bz);
	}
	return key;
}

// spread the low 21 bits of v to every third bit
__device__ __forceinline__ uint64_t spread3(uint64_t v)
{
	v &= 0x1FFFFFull;
	v = (v | (v << 32)) & 0x1F00000000FFFFull;
	v = (v | (v << 16)) & 0x1F0000FF0000FFull;
	v = (v | (v << 8)) & 0x100F00F00F00F00Full;
	v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
	v = (v | (v << 2)) & 0x1249249249249249ull;
	return v;
}

// Fast form: the same key layout from the scaled coordinate, cell j of level
// 21 being [j, j + 1) * w / 2^21; it differs from the midpoint descent only
// for points within rounding of a cell face, which the fast form tolerates.
__device__ __forceinline__ uint64_t scaled_key(double x, double y, double z, double scale)
{
	const double m = 2097151.0;
	const uint64_t ix = (uint64_t)fmin(fmax(x * scale, 0.0), m);
	const uint64_t iy = (uint64_t)fmin(fmax(y * scale, 0.0), m);
	const uint64_t iz = (uint64_t)fmin(fmax(z * scale, 0.0), m);
	return (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
}

// Keys of every particle (grid-stride) and, when hist is given, the digit
// counts of each of the radix sort's npass 8-bit passes from low_bit,
// hist[p * 256 + d], counted in shared memory and added once per block: the
// sort then needs no read of the keys of its own for them.
template <class G>
__device__ __forceinline__ void keys_body(G grd, const double4* __restrict__ pos, uint64_t* __restrict__ keys,
                                          uint32_t* __restrict__ vals, const Params& P, RunRec* rec, int begin_step,
                                          uint32_t* __restrict__ hist, int low_bit, int npass)
{
	__shared__ uint32_t h[OS_MAX_PASSES][RS_BINS];
	if (hist) {
		for (int i = threadIdx.x; i < npass * RS_BINS; i += blockDim.x) (&h[0][0])[i] = 0;
		__syncthreads();
	}
	if (begin_step && grd.id() == 0 && threadIdx.x == 0) {
		const unsigned long long t = rec->t_steps + 1;
		rec->t_steps = t;
		rec->n_due = 0;
		rec->n_rein = 0;
		rec->n_nodes = 0;
		rec->work_ctr = 0;
		rec->work_ctr2 = 0;
		rec->stack_max = 0;
		rec->grain_due = (t % P.tss[SP_DUST]) == 0 ? 1u : 0u;
		rec->dq = 0;
		rec->de = 0;
		rec->nabs_ion = 0;
		rec->nabs_e = 0;
		for (int k = 0; k < 3; k++) { rec->sumv_ion[k] = 0; rec->sumv_e[k] = 0; }
		rec->interactions = 0;
		rec->far_cells = 0;
		rec->n_pushed = 0;
		rec->n_collected = 0;
		rec->n_wall = 0;
		rec->n_bounced = 0;
		rec->grain_slot = 0xFFFFFFFFu;
	}
	for (uint32_t s = grd.id() * blockDim.x + threadIdx.x; s < P.n; s += grd.n() * blockDim.x) {
		const double4 p = pos[s];
		if (isnan(p.x) || isnan(p.y) || isnan(p.z)) {
			set_status(rec, POT_E_NONFINITE);
		} else if (p.x < 0.0 || p.x > P.root_w || p.y < 0.0 || p.y > P.root_w || p.z < 0.0 || p.z > P.root_w) {
			set_status(rec, POT_E_DOMAIN);  // build_tree returns NULL, pot.c:1491-1500
		}
		// A spheroidal grain is not a tree source (pot-spheroid.c:1516-1518): the
		// largest key sorts it to the last slot, outside [0, n_tree).  No
		// particle of the spherical domain lies in that corner cell.
		const uint64_t k = (P.shape && (int)p.w == SP_DUST) ? 0x7FFFFFFFFFFFFFFFull
		                   : P.form == POT_FORM_FAST       ? scaled_key(p.x, p.y, p.z, 2097152.0 / P.root_w)
		                                                   : morton_key(p.x, p.y, p.z, P.root_w);
		keys[s] = k;
		vals[s] = s;
		if (hist)
			for (int q = 0; q < npass; q++) atomicAdd(&h[q][(k >> (low_bit + 8 * q)) & 0xFF], 1u);
	}
	if (hist) {
		__syncthreads();
		for (int i = threadIdx.x; i < npass * RS_BINS; i += blockDim.x) {
			const uint32_t c = (&h[0][0])[i];
			if (c) atomicAdd(&hist[i], c);
		}
	}
}

__global__ void k_keys(const double4* __restrict__ pos, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                       Params P, RunRec* rec, int begin_step, uint32_t* __restrict__ hist, int low_bit, int npass)
{
	keys_body(GridSelf {}, pos, keys, vals, P, rec, begin_step, hist, low_bit, npass);
}

// Gather the state into the new Morton order, write the tree sources and
// mark the particles due this step (electrons every step, ions every
// tss[ION] steps, the grain every tss[DUST] steps, pot.c:2430-2434).
// One slot of the reorder; returns whether the particle is due.
__device__ __forceinline__ bool reorder_one(uint32_t s, const uint32_t* __restrict__ perm,
                                            const double4* __restrict__ pos_in, const double4* __restrict__ vel_in,
                                            const uint32_t* __restrict__ pid_in, double4* __restrict__ pos_out,
                                            double4* __restrict__ vel_out, uint32_t* __restrict__ pid_out,
                                            double4* __restrict__ src64, float4* __restrict__ src32,
                                            uint8_t* __restrict__ due, const Params& P, RunRec* rec)
{
	const uint32_t j = perm[s];
	const double4 p = pos_in[j];
	const double4 v = vel_in[j];
	const uint32_t id = pid_in[j];
	const int sp = (int)p.w;
	const double q = sp == SP_DUST ? (double)rec->grain_q : (sp == SP_ION ? 1.0 : -1.0);
	pos_out[s] = p;
	vel_out[s] = v;
	pid_out[s] = id;
	src64[s] = make_double4(p.x, p.y, p.z, q);
	if (src32) {
		src32[s] = make_float4((float)((p.x - P.rad) * P.inv_rad), (float)((p.y - P.rad) * P.inv_rad),
		                       (float)((p.z - P.rad) * P.inv_rad), (float)q);
	}
	const bool d = (rec->t_steps % P.tss[sp]) == 0;
	due[s] = d ? 1 : 0;
	if (sp == SP_DUST) rec->grain_slot = s;
	return d;
}


template <class G>
__device__ __forceinline__ void reorder_body(G grd, const uint32_t* __restrict__ perm,
                                             const double4* __restrict__ pos_in, const double4* __restrict__ vel_in,
                                             const uint32_t* __restrict__ pid_in, double4* __restrict__ pos_out,
                                             double4* __restrict__ vel_out, uint32_t* __restrict__ pid_out,
                                             double4* __restrict__ src64, float4* __restrict__ src32,
                                             uint8_t* __restrict__ due, const Params& P, RunRec* rec,
                                             uint32_t* __restrict__ due_tiles)
{
	const uint32_t s = grd.id() * blockDim.x + threadIdx.x;
	// the due flags' count per scan tile of SCAN_TILE slots (the compaction's
	// first stage; a 256-thread block lies inside one tile)
	bool is_due = false;
	if (s < P.n) is_due = reorder_one(s, perm, pos_in, vel_in, pid_in, pos_out, vel_out, pid_out, src64, src32, due,
	                                  P, rec);
	if (due_tiles) {
		__shared__ uint32_t wcnt[32];
		const uint32_t c = __popc(__ballot_sync(0xffffffffu, is_due));
		if ((threadIdx.x & 31) == 0) wcnt[threadIdx.x >> 5] = c;
		__syncthreads();
		if (threadIdx.x == 0) {
			uint32_t t = 0;
			for (uint32_t w = 0; w < (blockDim.x >> 5); w++) t += wcnt[w];
			if (t) atomicAdd(&due_tiles[(grd.id() * blockDim.x) / SCAN_TILE], t);
		}
	}
}

__global__ void k_reorder(const uint32_t* __restrict__ perm, const double4* __restrict__ pos_in,
                          const double4* __restrict__ vel_in, const uint32_t* __restrict__ pid_in,
                          double4* __restrict__ pos_out, double4* __restrict__ vel_out,
                          uint32_t* __restrict__ pid_out, double4* __restrict__ src64, float4* __restrict__ src32,
                          uint8_t* __restrict__ due, Params P, RunRec* rec, uint32_t* __restrict__ due_tiles)
{
	reorder_body(GridSelf {}, perm, pos_in, vel_in, pid_in, pos_out, vel_out, pid_out, src64, src32, due, P, rec,
	             due_tiles);
}

__device__ __forceinline__ int lcp_levels(uint64_t a, uint64_t b)
{
	const uint64_t x = a ^ b;
	if (x == 0) return MAX_LEVELS;
	return (__clzll((long long)x) - 1) / 3;
}

// lvl8[i] = common levels of keys i and i + L (capped at 20: a level-21
// cell cannot split); cnt[i] = number of cells pair i owns.
template <class G>
__device__ __forceinline__ void pairs_body(G grd, const uint64_t* __restrict__ keys,
                                           const double4* __restrict__ src64, uint32_t n, uint32_t n_pairs,
                                           uint32_t L, int max_level, int8_t* __restrict__ lvl8,
                                           uint32_t* __restrict__ cnt, RunRec* rec)
{
	const uint32_t i = grd.id() * blockDim.x + threadIdx.x;
	// Two particles at one position: the reference's insertion would split
	// forever (pot.c:1466-1470) or fail at a reallocation (pot.c:1578-1586).
	if (i + 1 < n && keys[i] == keys[i + 1]) {
		const double4 a = src64[i], b = src64[i + 1];
		if (a.x == b.x && a.y == b.y && a.z == b.z) set_status(rec, POT_E_COINCIDENT);
	}
	if (i >= n_pairs) return;
	const int li = lcp_levels(keys[i], keys[i + L]);
	if (li == MAX_LEVELS && max_level == MAX_LEVELS) atomicOr(&rec->warn, 1u);
	const int hi = li < max_level - 1 ? li : max_level - 1;
	int prev = -1;
	if (i > 0) {
		const int lp = lcp_levels(keys[i - 1], keys[i - 1 + L]);
		prev = lp < max_level - 1 ? lp : max_level - 1;
	}
	lvl8[i] = (int8_t)hi;
	cnt[i] = hi > prev ? (uint32_t)(hi - prev) : 0u;
}

__global__ void k_pairs(const uint64_t* __restrict__ keys, const double4* __restrict__ src64, uint32_t n,
                        uint32_t n_pairs, uint32_t L, int max_level, int8_t* __restrict__ lvl8,
                        uint32_t* __restrict__ cnt, RunRec* rec)
{
	pairs_body(GridSelf {}, keys, src64, n, n_pairs, L, max_level, lvl8, cnt, rec);
}

template <class G>
__device__ __forceinline__ void fill_nodes_body(G grd, const int8_t* __restrict__ lvl8,
                                                const uint32_t* __restrict__ base, uint32_t n_pairs, const TreeDev& T,
                                                RunRec* rec)
{
	const uint32_t i = grd.id() * blockDim.x + threadIdx.x;
	if (i >= n_pairs) return;
	const int hi = lvl8[i];
	const int lo = i == 0 ? 0 : lvl8[i - 1] + 1;
	for (int l = lo; l <= hi; l++) {
		const uint32_t k = base[i] + (uint32_t)(l - lo);
		if (k >= T.cap) {
			set_status(rec, POT_E_CAPACITY);
			return;
		}
		T.first[k] = i;
		T.level[k] = (uint8_t)l;
	}
}

__global__ void k_fill_nodes(const int8_t* __restrict__ lvl8, const uint32_t* __restrict__ base, uint32_t n_pairs,
                             TreeDev T, RunRec* rec)
{
	fill_nodes_body(GridSelf {}, lvl8, base, n_pairs, T, rec);
}

// The searches below run over a cell's sorted key range, where the tested
// property holds on a prefix of the range.  They make several independent
// reads per round, so that the chain of dependent loads -- which sets the
// time of the cells near the root -- is short.

// First index in [a, b) at which `pred` fails, b if it holds throughout:
// seven probes per round keep one eighth of the range; the last eight or
// fewer are read at once.
template <class Pred>
__device__ __forceinline__ uint32_t first_fail8(const uint64_t* __restrict__ keys, uint32_t a, uint32_t b, Pred pred)
{
	while (b - a > 8u) {
		const uint64_t span = b - a;
		uint32_t p[7];
		bool ok[7];
#pragma unroll
		for (int i = 0; i < 7; i++) p[i] = a + (uint32_t)((span * (uint64_t)(i + 1)) >> 3);  // a < p[0] < ... < p[6] < b
#pragma unroll
		for (int i = 0; i < 7; i++) ok[i] = pred(keys[p[i]]);
		uint32_t na = a, nb = b;
#pragma unroll
		for (int i = 0; i < 7; i++)
			if (ok[i]) na = p[i] + 1;  // the last probe that holds
#pragma unroll
		for (int i = 6; i >= 0; i--)
			if (!ok[i]) nb = p[i];  // the first probe that fails
		a = na;
		b = nb;
	}
	uint32_t c = 0;
#pragma unroll
	for (int i = 0; i < 8; i++) c += (a + (uint32_t)i < b && pred(keys[a + i])) ? 1u : 0u;
	return a + c;
}

// One past the last slot of the cell that starts at slot f with key prefix
// pfx (key >> shift): f + 2^e is probed for seven exponents per round until
// one leaves the cell, then the bracket is searched.
__device__ __forceinline__ uint32_t cell_end(const uint64_t* __restrict__ keys, uint32_t f, uint32_t n, int shift,
                                             uint64_t pfx)
{
	const auto same = [=](uint64_t k) { return (k >> shift) == pfx; };
	uint32_t a = f + 1, b = n;
	for (int e0 = 0; e0 < 32; e0 += 7) {
		uint64_t q[7];
		bool ok[7];
#pragma unroll
		for (int i = 0; i < 7; i++) {
			q[i] = (uint64_t)f + (1ull << (e0 + i));
			ok[i] = q[i] < n && same(keys[q[i]]);
		}
		bool left = false;
#pragma unroll
		for (int i = 0; i < 7; i++)
			if (ok[i]) a = (uint32_t)q[i] + 1;
#pragma unroll
		for (int i = 6; i >= 0; i--) {
			if (!ok[i]) {
				b = q[i] < n ? (uint32_t)q[i] : n;
				left = true;
			}
		}
		if (left) break;
	}
	return first_fail8(keys, a, b, same);
}

// s[c] for c = 1..7: the first slot of [f, e) whose child digit at `shift`
// is >= c; seven bisections side by side.
__device__ __forceinline__ void child_starts(const uint64_t* __restrict__ keys, uint32_t f, uint32_t e, int shift,
                                             uint32_t s[9])
{
	uint32_t lo[7], hi[7];
#pragma unroll
	for (int c = 0; c < 7; c++) {
		lo[c] = f;
		hi[c] = e;
	}
	for (uint32_t span = e - f; span > 0u; span >>= 1) {
#pragma unroll
		for (int c = 0; c < 7; c++) {
			if (lo[c] < hi[c]) {
				const uint32_t m = lo[c] + ((hi[c] - lo[c]) >> 1);
				if (((keys[m] >> shift) & 7u) < (uint32_t)(c + 1)) lo[c] = m + 1; else hi[c] = m;
			}
		}
	}
#pragma unroll
	for (int c = 0; c < 7; c++) s[c + 1] = lo[c];
}

template <class G>
__device__ __forceinline__ void finish_nodes_body(G grd, const uint64_t* __restrict__ keys, uint32_t n, uint32_t L,
                                                  const int8_t* __restrict__ lvl8, const uint32_t* __restrict__ base,
                                                  const TreeDev& T, const Params& P, RunRec* rec)
{
	const uint32_t M = rec->n_nodes;
	if (M > T.cap) {
		if (grd.id() == 0 && threadIdx.x == 0) set_status(rec, POT_E_CAPACITY);
		return;
	}
	for (uint32_t k = grd.id() * blockDim.x + threadIdx.x; k < M; k += grd.n() * blockDim.x) {
		const uint32_t f = T.first[k];
		const int l = T.level[k];
		const int shift = 63 - 3 * l;
		const uint64_t pfx = keys[f] >> shift;
		// last particle of the cell
		const uint32_t last = cell_end(keys, f, n, shift, pfx) - 1;
		T.last[k] = last;
		// children by digit at the next level
		const int cshift = shift - 3;
		uint32_t s[9];
		s[0] = f;
		s[8] = last + 1;
		child_starts(keys, f, last + 1, cshift, s);
		int nint = 0;
#pragma unroll
		for (int c = 0; c < 8; c++) {
			const uint32_t cnt = s[c + 1] - s[c];
			int32_t code;
			if (cnt == 0) {
				code = CH_EMPTY;
			} else if (cnt <= L || l + 1 >= (int)P.max_level) {
				if (L == 1 && cnt == 1) {
					code = leaf_code(s[c]);
				} else if (L == 1) {
					const uint32_t j = atomicAdd(&rec->n_overflow, 1u);
					atomicOr(&rec->warn, 1u);
					if (j < OVF_CAP) {
						T.ovf[j] = make_uint2(s[c], cnt);
						code = leaf_code(n + j);
					} else {
						set_status(rec, POT_E_CAPACITY);
						code = CH_EMPTY;
					}
				} else {
					const uint32_t e = 8u * k + (uint32_t)c;
					code = leaf_code(e);
					T.lrange[e] = make_uint2(s[c], cnt);
				}
			} else {
				const uint32_t sc = s[c];
				const int lo = sc == 0 ? 0 : lvl8[sc - 1] + 1;
				const uint32_t kc = base[sc] + (uint32_t)(l + 1 - lo);
				if (sc + L >= n || kc >= M || kc <= k) {
					// cannot happen for a consistent key order; never write out of range
					set_status(rec, POT_E_CAPACITY);
					code = CH_EMPTY;
				} else {
					code = (int32_t)kc;
					T.parent[kc] = (int32_t)k;
					nint++;
				}
			}
			T.child[8u * k + (uint32_t)c] = code;
		}
		T.nint[k] = (uint8_t)nint;
		T.ctr[k] = 0;
		if (k == 0) T.parent[0] = -1;
		// x-extent of the cell by the reference's halving (pot.c:1262)
		double lo = 0.0, hi = P.root_w;
		for (int lev = 1; lev <= l; lev++) {
			const uint32_t bit = (uint32_t)(pfx >> (3 * (l - lev) + 2)) & 1u;
			const double mid = dmul(dadd(lo, hi), 0.5);
			if (bit) lo = mid; else hi = mid;
		}
		const double w = dsub(hi, lo);
		T.w2[k] = dmul(w, w);
	}
}

__global__ void k_finish_nodes(const uint64_t* __restrict__ keys, uint32_t n, uint32_t L,
                               const int8_t* __restrict__ lvl8, const uint32_t* __restrict__ base, TreeDev T,
                               Params P, RunRec* rec)
{
	finish_nodes_body(GridSelf {}, keys, n, L, lvl8, base, T, P, rec);
}

// running |q|-weighted update of pot.c:1290-1310
__device__ __forceinline__ void add_moment(int& q, uint32_t& aq, double& cx, double& cy, double& cz, int cq,
                                           uint32_t caq, double ccx, double ccy, double ccz)
{
	const double a0 = (double)aq, a1 = (double)caq, den = (double)(aq + caq);
	cx = ddiv(dadd(dmul(a0, cx), dmul(a1, ccx)), den);
	cy = ddiv(dadd(dmul(a0, cy), dmul(a1, ccy)), den);
	cz = ddiv(dadd(dmul(a0, cz), dmul(a1, ccz)), den);
	q += cq;
	aq += caq;
}

// DIPOLES (pot.c:1290-1310): the node's dipole moves to the new centre of
// |q|, then the child's, moved there too, is added; q and |q| last
__device__ __forceinline__ void add_moment_dip(int& q, uint32_t& aq, double& cx, double& cy, double& cz, double& px,
                                               double& py, double& pz, int cq, uint32_t caq, double ccx, double ccy,
                                               double ccz, double cpx, double cpy, double cpz)
{
	const double ox = cx, oy = cy, oz = cz;
	const double a0 = (double)aq, a1 = (double)caq, den = (double)(aq + caq);
	cx = ddiv(dadd(dmul(a0, cx), dmul(a1, ccx)), den);
	cy = ddiv(dadd(dmul(a0, cy), dmul(a1, ccy)), den);
	cz = ddiv(dadd(dmul(a0, cz), dmul(a1, ccz)), den);
	const double qd = (double)q, cqd = (double)cq;
	px = dsub(px, dmul(dsub(cx, ox), qd));
	py = dsub(py, dmul(dsub(cy, oy), qd));
	pz = dsub(pz, dmul(dsub(cz, oz), qd));
	px = dadd(px, dsub(cpx, dmul(dsub(cx, ccx), cqd)));
	py = dadd(py, dsub(cpy, dmul(dsub(cy, ccy), cqd)));
	pz = dadd(pz, dsub(cpz, dmul(dsub(cz, ccz), cqd)));
	q += cq;
	aq += caq;
}

__global__ void k_moments(TreeDev T, const double4* __restrict__ src64, Params P, RunRec* rec)
{
	const uint32_t M = rec->n_nodes;
	if (M > T.cap) return;
	const uint32_t L = P.leaf_size;
	const bool dip = T.dip != nullptr;
	for (uint32_t k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < M; k0 += gridDim.x * blockDim.x) {
	if (T.nint[k0] != 0) continue;
	uint32_t k = k0;
	for (;;) {
		int q = 0;
		uint32_t aq = 0;
		double cx = 0.0, cy = 0.0, cz = 0.0;
		double px = 0.0, py = 0.0, pz = 0.0;
		const float w_child = 0.5f * (float)(sqrt(T.w2[k]) * P.inv_rad);
		for (int s = 0; s < 8; s++) {
			const int d = slot_digit(s);
			const int32_t code = T.child[8u * k + (uint32_t)d];
			if (code == CH_EMPTY) continue;
			int cq;
			uint32_t caq;
			double ccx, ccy, ccz;
			double cpx = 0.0, cpy = 0.0, cpz = 0.0;
			if (code >= 0) {
				cq = __ldcg(&T.q[code]);
				caq = __ldcg(&T.aq[code]);
				const double2* cp2 = reinterpret_cast<const double2*>(&T.cq[code]);
				const double2 c01 = __ldcg(cp2), c23 = __ldcg(cp2 + 1);
				const double4 c = make_double4(c01.x, c01.y, c23.x, c23.y);
				ccx = c.x; ccy = c.y; ccz = c.z;
				if (dip) {
					const double2* dp2 = reinterpret_cast<const double2*>(&T.dip[code]);
					const double2 d01 = __ldcg(dp2), d23 = __ldcg(dp2 + 1);
					cpx = d01.x; cpy = d01.y; cpz = d23.x;
				}
			} else if (L == 1 && leaf_payload(code) < P.n_tree) {
				const double4 sp = src64[leaf_payload(code)];
				cq = (int)sp.w;
				caq = (uint32_t)abs(cq);
				ccx = sp.x; ccy = sp.y; ccz = sp.z;
			} else {
				// bucket leaf: its own running moments over its particles
				const uint32_t e = leaf_payload(code);
				const uint2 r = L == 1 ? T.ovf[e - P.n_tree] : T.lrange[e];
				cq = 0;
				caq = 0;
				ccx = ccy = ccz = 0.0;
				for (uint32_t j = r.x; j < r.x + r.y; j++) {
					const double4 sp = src64[j];
					const int pq = (int)sp.w;
					const uint32_t paq = (uint32_t)abs(pq);
					if (!paq) continue;
					if (dip) {
						add_moment_dip(cq, caq, ccx, ccy, ccz, cpx, cpy, cpz, pq, paq, sp.x, sp.y, sp.z, 0.0, 0.0,
						               0.0);
					} else {
						add_moment(cq, caq, ccx, ccy, ccz, pq, paq, sp.x, sp.y, sp.z);
					}
				}
				if (T.lf && L > 1) {
					T.lf[e] = make_float4((float)((ccx - P.rad) * P.inv_rad), (float)((ccy - P.rad) * P.inv_rad),
					                      (float)((ccz - P.rad) * P.inv_rad), (float)cq);
					T.lr2[e] = w_child * w_child / P.oap2_f;
				}
			}
			if (caq) {
				if (dip) {
					add_moment_dip(q, aq, cx, cy, cz, px, py, pz, cq, caq, ccx, ccy, ccz, cpx, cpy, cpz);
				} else {
					add_moment(q, aq, cx, cy, cz, cq, caq, ccx, ccy, ccz);
				}
			}
		}
		T.q[k] = q;
		T.aq[k] = aq;
		T.cq[k] = make_double4(cx, cy, cz, (double)q);
		if (dip) T.dip[k] = make_double4(px, py, pz, 0.0);
		if (T.f) {
			T.f[k] = make_float4((float)((cx - P.rad) * P.inv_rad), (float)((cy - P.rad) * P.inv_rad),
			                     (float)((cz - P.rad) * P.inv_rad), (float)q);
			T.r2[k] = (float)(T.w2[k] * P.inv_rad * P.inv_rad / P.oap2);
		}
		if (k == 0) break;
		const int32_t p = T.parent[k];
		if (p < 0 || (uint32_t)p >= k) {  // parents precede children in pre-order
			set_status(rec, POT_E_CAPACITY);
			break;
		}
		__threadfence();
		const uint32_t arrived = atomicAdd(&T.ctr[p], 1u) + 1u;
		if (arrived != T.nint[p]) break;
		__threadfence();
		k = (uint32_t)p;
	}
	}
}

// Fast form: the same bottom-up pass with plain sums, sum |q| x / sum |q|
// divided once per cell, and bucket leaves summed directly.
__global__ void k_moments_fast(TreeDev T, const double4* __restrict__ src64, Params P, RunRec* rec)
{
	const uint32_t M = rec->n_nodes;
	if (M > T.cap) return;
	const uint32_t L = P.leaf_size;
	for (uint32_t k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < M; k0 += gridDim.x * blockDim.x) {
		if (T.nint[k0] != 0) continue;
		uint32_t k = k0;
		for (;;) {
			int q = 0;
			uint32_t aq = 0;
			double sx = 0.0, sy = 0.0, sz = 0.0;
			const float w_child = 0.5f * (float)(sqrt(T.w2[k]) * P.inv_rad);
			const int4* cp = reinterpret_cast<const int4*>(&T.child[8u * k]);
			const int4 c0 = cp[0], c1 = cp[1];
			const int32_t cc[8] = { c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w };
#pragma unroll
			for (int d = 0; d < 8; d++) {
				const int32_t code = cc[d];
				if (code == CH_EMPTY) continue;
				if (code >= 0) {
					const int cq = __ldcg(&T.q[code]);
					const uint32_t caq = __ldcg(&T.aq[code]);
					const double2* p2 = reinterpret_cast<const double2*>(&T.cq[code]);
					const double2 a01 = __ldcg(p2), a23 = __ldcg(p2 + 1);
					q += cq;
					aq += caq;
					sx = fma((double)caq, a01.x, sx);
					sy = fma((double)caq, a01.y, sy);
					sz = fma((double)caq, a23.x, sz);
					continue;
				}
				const uint32_t e = leaf_payload(code);
				uint32_t j0 = e, j1 = e + 1;
				if (L > 1) {
					const uint2 r = T.lrange[e];
					j0 = r.x;
					j1 = r.x + r.y;
				} else if (e >= P.n_tree) {
					const uint2 r = T.ovf[e - P.n_tree];
					j0 = r.x;
					j1 = r.x + r.y;
				}
				int lq = 0;
				uint32_t laq = 0;
				double lx = 0.0, ly = 0.0, lz = 0.0;
				for (uint32_t j = j0; j < j1; j++) {
					const double4 sp = src64[j];
					const int pq = (int)sp.w;
					const double pa = (double)abs(pq);
					lq += pq;
					laq += (uint32_t)abs(pq);
					lx = fma(pa, sp.x, lx);
					ly = fma(pa, sp.y, ly);
					lz = fma(pa, sp.z, lz);
				}
				if (L > 1 && T.lf) {
					const double inv = laq ? 1.0 / (double)laq : 0.0;
					T.lf[e] = make_float4((float)((lx * inv - P.rad) * P.inv_rad), (float)((ly * inv - P.rad) * P.inv_rad),
					                      (float)((lz * inv - P.rad) * P.inv_rad), (float)lq);
					T.lr2[e] = w_child * w_child / P.oap2_f;
				}
				q += lq;
				aq += laq;
				sx += lx;
				sy += ly;
				sz += lz;
			}
			const double inv = aq ? 1.0 / (double)aq : 0.0;
			const double cx = sx * inv, cy = sy * inv, cz = sz * inv;
			T.q[k] = q;
			T.aq[k] = aq;
			T.cq[k] = make_double4(cx, cy, cz, (double)q);
			T.f[k] = make_float4((float)((cx - P.rad) * P.inv_rad), (float)((cy - P.rad) * P.inv_rad),
			                     (float)((cz - P.rad) * P.inv_rad), (float)q);
			T.r2[k] = (float)(T.w2[k] * P.inv_rad * P.inv_rad / P.oap2);
			if (k == 0) break;
			const int32_t p = T.parent[k];
			if (p < 0 || (uint32_t)p >= k) {
				set_status(rec, POT_E_CAPACITY);
				break;
			}
			__threadfence();
			const uint32_t arrived = atomicAdd(&T.ctr[p], 1u) + 1u;
			if (arrived != T.nint[p]) break;
			__threadfence();
			k = (uint32_t)p;
		}
	}
}

// ---------------------------------------------------------------------------
// Fast form moments from prefix sums.  With particles in Morton order every
// cell and bucket leaf is a contiguous slot range [a, b), so its net charge,
// absolute charge and |q|-weighted position sums are differences of
// exclusive prefix sums P[b] - P[a] of (q, |q|, |q|(x - c), |q|(y - c),
// |q|(z - c)), c the domain centre.  FP64 sums: with |x - c| <= R the
// cancellation error of a difference is ~1e-16 of the largest prefix, far
// below the FP32 resolution the fast walk uses.
// ---------------------------------------------------------------------------
struct Mom5 {
	double q, a, x, y, z;
};

__device__ __forceinline__ Mom5 mom_add(const Mom5& u, const Mom5& v)
{
	return Mom5 { u.q + v.q, u.a + v.a, u.x + v.x, u.y + v.y, u.z + v.z };
}

// K = 0: (q, |q|, |q| x, |q| y, |q| z); K = 1 (DIPOLES): (q x, q y, q z, 0, 0);
// positions relative to the domain centre c
template <int K>
__device__ __forceinline__ Mom5 mom_of(const double4& p, double c)
{
	if (K == 1) return Mom5 { p.w * (p.x - c), p.w * (p.y - c), p.w * (p.z - c), 0.0, 0.0 };
	const double a = fabs(p.w);
	return Mom5 { p.w, a, a * (p.x - c), a * (p.y - c), a * (p.z - c) };
}

__device__ __forceinline__ Mom5 mom_shfl_up(const Mom5& m, int o)
{
	return Mom5 { __shfl_up_sync(0xffffffffu, m.q, o), __shfl_up_sync(0xffffffffu, m.a, o),
	              __shfl_up_sync(0xffffffffu, m.x, o), __shfl_up_sync(0xffffffffu, m.y, o),
	              __shfl_up_sync(0xffffffffu, m.z, o) };
}

constexpr int MOM_THREADS = 256;
constexpr int MOM_ITEMS = 16;
constexpr int MOM_TILE = MOM_THREADS * MOM_ITEMS;

// exclusive block scan of one Mom5 per thread; *tot = block total
__device__ Mom5 mom_block_excl(Mom5 v, Mom5* tot)
{
	__shared__ Mom5 wsum[MOM_THREADS / 32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	Mom5 inc = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const Mom5 t = mom_shfl_up(inc, o);
		if (lane >= o) inc = mom_add(inc, t);
	}
	if (lane == 31) wsum[w] = inc;
	__syncthreads();
	if (threadIdx.x == 0) {
		Mom5 run = Mom5 { 0, 0, 0, 0, 0 };
		for (int k = 0; k < MOM_THREADS / 32; k++) {
			const Mom5 t = wsum[k];
			wsum[k] = run;
			run = mom_add(run, t);
		}
		*tot = run;
	}
	__syncthreads();
	const Mom5 excl = mom_add(wsum[w], Mom5 { inc.q - v.q, inc.a - v.a, inc.x - v.x, inc.y - v.y, inc.z - v.z });
	__syncthreads();
	return excl;
}

// Each warp owns a contiguous chunk of MOM_ITEMS * 32 particles of the tile
// and walks it 32 at a time (coalesced loads).
__device__ __forceinline__ Mom5 mom_warp_incl(Mom5 v)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const Mom5 t = mom_shfl_up(v, o);
		if (lane >= o) v = mom_add(v, t);
	}
	return v;
}

__device__ __forceinline__ Mom5 mom_shfl(const Mom5& m, int src)
{
	return Mom5 { __shfl_sync(0xffffffffu, m.q, src), __shfl_sync(0xffffffffu, m.a, src),
	              __shfl_sync(0xffffffffu, m.x, src), __shfl_sync(0xffffffffu, m.y, src),
	              __shfl_sync(0xffffffffu, m.z, src) };
}

template <int K, class G>
__device__ __forceinline__ void mom_reduce_body(G grd, const double4* __restrict__ src64, uint32_t n, double c,
                                                Mom5* __restrict__ bsum)
{
	__shared__ Mom5 tot;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const size_t base = (size_t)grd.id() * MOM_TILE + (size_t)w * (MOM_ITEMS * 32);
	Mom5 s = Mom5 { 0, 0, 0, 0, 0 };
	for (int k = 0; k < MOM_ITEMS; k++) {
		const size_t i = base + (size_t)k * 32 + lane;
		if (i < n) s = mom_add(s, mom_of<K>(src64[i], c));
	}
	mom_block_excl(s, &tot);
	if (threadIdx.x == 0) bsum[grd.id()] = tot;
}

template <int K>
__global__ void __launch_bounds__(MOM_THREADS) k_mom_reduce(const double4* __restrict__ src64, uint32_t n, double c,
                                                            Mom5* __restrict__ bsum)
{
	mom_reduce_body<K>(GridSelf {}, src64, n, c, bsum);
}

template <class G>
__device__ __forceinline__ void mom_top_body(G grd, Mom5* __restrict__ bsum, uint32_t nb)
{
	__shared__ Mom5 tot;
	__shared__ Mom5 carry;
	if (threadIdx.x == 0) carry = Mom5 { 0, 0, 0, 0, 0 };
	__syncthreads();
	for (uint32_t base = 0; base < nb; base += MOM_THREADS) {
		const uint32_t i = base + threadIdx.x;
		const Mom5 v = i < nb ? bsum[i] : Mom5 { 0, 0, 0, 0, 0 };
		const Mom5 e = mom_block_excl(v, &tot);
		const Mom5 c = carry;
		if (i < nb) bsum[i] = mom_add(c, e);
		__syncthreads();
		if (threadIdx.x == 0) carry = mom_add(c, tot);
		__syncthreads();
	}
}

__global__ void __launch_bounds__(MOM_THREADS) k_mom_top(Mom5* __restrict__ bsum, uint32_t nb)
{
	mom_top_body(GridSelf {}, bsum, nb);
}

template <int K, class G>
__device__ __forceinline__ void mom_down_body(G grd, const double4* __restrict__ src64, uint32_t n, double c,
                                              const Mom5* __restrict__ bsum, Mom5* __restrict__ pre)
{
	__shared__ Mom5 tot;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const size_t base = (size_t)grd.id() * MOM_TILE + (size_t)w * (MOM_ITEMS * 32);
	// this warp's chunk total, then its offset among the block's warps
	Mom5 s = Mom5 { 0, 0, 0, 0, 0 };
	for (int k = 0; k < MOM_ITEMS; k++) {
		const size_t i = base + (size_t)k * 32 + lane;
		if (i < n) s = mom_add(s, mom_of<K>(src64[i], c));
	}
	// reduce the per-lane partial sums to the warp total on lane 0
	Mom5 wt = s;
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		wt = mom_add(wt, Mom5 { __shfl_xor_sync(0xffffffffu, wt.q, o), __shfl_xor_sync(0xffffffffu, wt.a, o),
		                        __shfl_xor_sync(0xffffffffu, wt.x, o), __shfl_xor_sync(0xffffffffu, wt.y, o),
		                        __shfl_xor_sync(0xffffffffu, wt.z, o) });
	}
	const Mom5 mine = lane == 0 ? wt : Mom5 { 0, 0, 0, 0, 0 };
	Mom5 carry = mom_add(bsum[grd.id()], mom_block_excl(mine, &tot));  // valid on lane 0
	carry = mom_shfl(carry, 0);
	for (int k = 0; k < MOM_ITEMS; k++) {
		const size_t i = base + (size_t)k * 32 + lane;
		const Mom5 v = i < n ? mom_of<K>(src64[i], c) : Mom5 { 0, 0, 0, 0, 0 };
		const Mom5 inc = mom_warp_incl(v);
		if (i < n) {
			pre[i] = mom_add(carry, Mom5 { inc.q - v.q, inc.a - v.a, inc.x - v.x, inc.y - v.y, inc.z - v.z });
			if (i + 1 == n) pre[n] = mom_add(carry, inc);
		}
		carry = mom_add(carry, mom_shfl(inc, 31));
	}
}

template <int K>
__global__ void __launch_bounds__(MOM_THREADS) k_mom_down(const double4* __restrict__ src64, uint32_t n, double c,
                                                          const Mom5* __restrict__ bsum, Mom5* __restrict__ pre)
{
	mom_down_body<K>(GridSelf {}, src64, n, c, bsum, pre);
}

__device__ __forceinline__ Mom5 mom_range(const Mom5* __restrict__ pre, uint32_t a, uint32_t b)
{
	const Mom5 u = pre[b], v = pre[a];
	return Mom5 { u.q - v.q, u.a - v.a, u.x - v.x, u.y - v.y, u.z - v.z };
}

// DIPOLES: the dipole about the centre of |q| from the prefix sums of q x
// (pd) and the cell's charge and centre (relative to the domain centre),
// p = sum q (x - c) = sum q x - Q c
__device__ __forceinline__ double3 dipole_of(const Mom5& pd, double q, double cx, double cy, double cz)
{
	return make_double3(pd.q - q * cx, pd.a - q * cy, pd.x - q * cz);
}

template <class G>
__device__ __forceinline__ void moments_prefix_body(G grd, const TreeDev& T, const Mom5* __restrict__ pre,
                                                    const Mom5* __restrict__ pre_d, const Params& P, RunRec* rec)
{
	const uint32_t M = rec->n_nodes;
	if (M > T.cap) return;
	const uint32_t L = P.leaf_size;
	for (uint32_t k = grd.id() * blockDim.x + threadIdx.x; k < M; k += grd.n() * blockDim.x) {
		const Mom5 m = mom_range(pre, T.first[k], T.last[k] + 1);
		const double inv = m.a > 0.0 ? 1.0 / m.a : 0.0;
		const double cx = m.x * inv, cy = m.y * inv, cz = m.z * inv;  // relative to the centre
		const int q = (int)llrint(m.q);
		T.q[k] = q;
		T.aq[k] = (uint32_t)llrint(m.a);
		T.cq[k] = make_double4(cx + P.rad, cy + P.rad, cz + P.rad, (double)q);
		T.f[k] = make_float4((float)(cx * P.inv_rad), (float)(cy * P.inv_rad), (float)(cz * P.inv_rad), (float)q);
		T.r2[k] = (float)(T.w2[k] * P.inv_rad * P.inv_rad / P.oap2);
		if (pre_d) {
			const double3 d = dipole_of(mom_range(pre_d, T.first[k], T.last[k] + 1), (double)q, cx, cy, cz);
			T.dip[k] = make_double4(d.x, d.y, d.z, 0.0);
			T.fd[k] = make_float4((float)(d.x * P.inv_rad), (float)(d.y * P.inv_rad), (float)(d.z * P.inv_rad), 0.f);
		}
		if (L > 1) {
			const float w_child = 0.5f * (float)(sqrt(T.w2[k]) * P.inv_rad);
			for (int d = 0; d < 8; d++) {
				const int32_t code = T.child[8u * k + (uint32_t)d];
				if (code >= CH_EMPTY) continue;
				const uint32_t e = leaf_payload(code);
				const uint2 r = T.lrange[e];
				const Mom5 lm = mom_range(pre, r.x, r.x + r.y);
				const double li = lm.a > 0.0 ? 1.0 / lm.a : 0.0;
				T.lf[e] = make_float4((float)(lm.x * li * P.inv_rad), (float)(lm.y * li * P.inv_rad),
				                      (float)(lm.z * li * P.inv_rad), (float)llrint(lm.q));
				T.lr2[e] = w_child * w_child / P.oap2_f;
				if (pre_d) {
					const double3 d = dipole_of(mom_range(pre_d, r.x, r.x + r.y), (double)llrint(lm.q), lm.x * li,
					                            lm.y * li, lm.z * li);
					T.lfd[e] = make_float4((float)(d.x * P.inv_rad), (float)(d.y * P.inv_rad),
					                       (float)(d.z * P.inv_rad), 0.f);
				}
			}
		}
	}
}

__global__ void k_moments_prefix(TreeDev T, const Mom5* __restrict__ pre, const Mom5* __restrict__ pre_d, Params P,
                                 RunRec* rec)
{
	moments_prefix_body(GridSelf {}, T, pre, pre_d, P, rec);
}

size_t mom_prefix_entries(size_t n) { return n + 1; }
size_t mom_block_entries(size_t n) { return (n + MOM_TILE - 1) / MOM_TILE + 1; }

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static inline uint32_t blocks_for(size_t n, int threads) { return (uint32_t)((n + threads - 1) / threads); }

// The keys kernel's grid: a block per 256 particles up to eight blocks per
// SM, then grid-stride (each block adds its digit counts once).
uint32_t keys_blocks(size_t n) { return std::min<uint32_t>(blocks_for(n, 256), 148u * 8u); }

void launch_keys(const double4* pos, uint64_t* keys, uint32_t* vals, const Params& P, RunRec* rec,
                 int begin_step, uint32_t* hist, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "keys");
	k_keys<<<keys_blocks(P.n), 256, 0, s>>>(pos, keys, vals, P, rec, begin_step, hist, (int)P.key_bits,
	                                        radix_passes((int)P.key_bits));
}

void launch_reorder(const uint32_t* perm, const double4* pos_in, const double4* vel_in, const uint32_t* pid_in,
                    double4* pos_out, double4* vel_out, uint32_t* pid_out, double4* src64, float4* src32,
                    uint8_t* due, const Params& P, RunRec* rec, uint32_t* due_tiles, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "reorder");
	k_reorder<<<blocks_for(P.n, 256), 256, 0, s>>>(perm, pos_in, vel_in, pid_in, pos_out, vel_out, pid_out,
	                                               src64, src32, due, P, rec, due_tiles);
}

void launch_build(const uint64_t* keys, TreeDev& T, const double4* src64, const Params& P, RunRec* rec,
                  uint32_t* block_sums, cudaStream_t s, Timer& tm)
{
	const uint32_t n = P.n_tree, L = P.leaf_size;
	const uint32_t n_pairs = n - L;  // n_tree > L is checked at creation
	cudaMemsetAsync(&rec->n_overflow, 0, sizeof(unsigned int), s);
	{
		ScopedKernel k(tm, "tree_pairs");
		k_pairs<<<blocks_for(n - 1, 256), 256, 0, s>>>(keys, src64, n, n_pairs, L, (int)P.max_level, T.lvl8,
		                                               T.cnt, rec);
	}
	scan_exclusive(T.cnt, T.base, n_pairs, block_sums, &rec->n_nodes, s, tm);
	{
		ScopedKernel k(tm, "tree_fill");
		k_fill_nodes<<<blocks_for(n_pairs, 256), 256, 0, s>>>(T.lvl8, T.base, n_pairs, T, rec);
	}
	{
		ScopedKernel k(tm, "tree_finish");
		k_finish_nodes<<<blocks_for(n, 256), 256, 0, s>>>(keys, n, L, T.lvl8, T.base, T, P, rec);
	}
	{
		const bool prefix = P.form == POT_FORM_FAST && T.mom_pre;
		const bool dip = prefix && T.mom_pre_d;
		ScopedKernel k(tm, "tree_moments", prefix ? (dip ? 7 : 4) : 1);
		if (prefix) {
			const uint32_t nb = (uint32_t)((n + MOM_TILE - 1) / MOM_TILE);
			Mom5* pre = reinterpret_cast<Mom5*>(T.mom_pre);
			Mom5* bs = reinterpret_cast<Mom5*>(T.mom_blk);
			k_mom_reduce<0><<<nb, MOM_THREADS, 0, s>>>(src64, n, P.rad, bs);
			k_mom_top<<<1, MOM_THREADS, 0, s>>>(bs, nb);
			k_mom_down<0><<<nb, MOM_THREADS, 0, s>>>(src64, n, P.rad, bs, pre);
			Mom5* pre_d = nullptr;
			if (dip) {  // DIPOLES: prefix sums of q x as well
				pre_d = reinterpret_cast<Mom5*>(T.mom_pre_d);
				Mom5* bs_d = reinterpret_cast<Mom5*>(T.mom_blk_d);
				k_mom_reduce<1><<<nb, MOM_THREADS, 0, s>>>(src64, n, P.rad, bs_d);
				k_mom_top<<<1, MOM_THREADS, 0, s>>>(bs_d, nb);
				k_mom_down<1><<<nb, MOM_THREADS, 0, s>>>(src64, n, P.rad, bs_d, pre_d);
			}
			k_moments_prefix<<<blocks_for(n / 4 + 1, 256), 256, 0, s>>>(T, pre, pre_d, P, rec);
		} else if (P.form == POT_FORM_FAST) {
			k_moments_fast<<<blocks_for(n, 256), 256, 0, s>>>(T, src64, P, rec);
		} else {
			k_moments<<<blocks_for(n, 256), 256, 0, s>>>(T, src64, P, rec);
		}
	}
}

}  // namespace pot

// ---------------------------------------------------------------------------
// packed batch: the same kernels, one launch over every member
// ---------------------------------------------------------------------------
namespace pot {

__global__ void kp_keys(PackDev B, int k)
{
	const SegBlock sb = seg_block(B.pre[PS_KEYS], B.M);
	const MemberView& v = B.mv[sb.m];
	keys_body(GridSeg { sb.id, sb.n }, v.pos[pack_in(v, k)], v.keys[0], v.vals[0], v.P, v.rec, 1,
	          v.counts + (size_t)OS_MAX_PASSES * v.tiles * RS_BINS, (int)v.P.key_bits, (int)B.npass);
}

__global__ void kp_reorder(PackDev B, int k)
{
	const SegBlock sb = seg_block(B.pre[PS_N256], B.M);
	const MemberView& v = B.mv[sb.m];
	const uint32_t a = pack_in(v, k), b = pack_out(v, k);
	reorder_body(GridSeg { sb.id, sb.n }, v.vals[v.kb], v.pos[a], v.vel[a], v.pid[a], v.pos[b], v.vel[b], v.pid[b],
	             v.src64, v.src32, v.due, v.P, v.rec, v.due_tiles);
}

__global__ void kp_pairs(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_PAIRS], B.M);
	const MemberView& v = B.mv[sb.m];
	const uint32_t n = v.P.n_tree, L = v.P.leaf_size;
	pairs_body(GridSeg { sb.id, sb.n }, v.keys[v.kb], v.src64, n, n - L, L, (int)v.P.max_level, v.T.lvl8, v.T.cnt,
	           v.rec);
}

__global__ void kp_fill_nodes(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_FILL], B.M);
	const MemberView& v = B.mv[sb.m];
	fill_nodes_body(GridSeg { sb.id, sb.n }, v.T.lvl8, v.T.base, v.P.n_tree - v.P.leaf_size, v.T, v.rec);
}

__global__ void kp_finish_nodes(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_FINISH], B.M);
	const MemberView& v = B.mv[sb.m];
	finish_nodes_body(GridSeg { sb.id, sb.n }, v.keys[v.kb], v.P.n_tree, v.P.leaf_size, v.T.lvl8, v.T.base, v.T,
	                  v.P, v.rec);
}

__global__ void __launch_bounds__(MOM_THREADS) kp_mom_reduce(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_MOM], B.M);
	const MemberView& v = B.mv[sb.m];
	mom_reduce_body<0>(GridSeg { sb.id, sb.n }, v.src64, v.P.n_tree, v.P.rad, reinterpret_cast<Mom5*>(v.T.mom_blk));
}

__global__ void __launch_bounds__(MOM_THREADS) kp_mom_top(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_ONE], B.M);
	const MemberView& v = B.mv[sb.m];
	const uint32_t nb = (v.P.n_tree + MOM_TILE - 1) / MOM_TILE;
	mom_top_body(GridSeg { sb.id, sb.n }, reinterpret_cast<Mom5*>(v.T.mom_blk), nb);
}

__global__ void __launch_bounds__(MOM_THREADS) kp_mom_down(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_MOM], B.M);
	const MemberView& v = B.mv[sb.m];
	mom_down_body<0>(GridSeg { sb.id, sb.n }, v.src64, v.P.n_tree, v.P.rad, reinterpret_cast<Mom5*>(v.T.mom_blk),
	                 reinterpret_cast<Mom5*>(v.T.mom_pre));
}

__global__ void kp_moments_prefix(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_MOMPRE], B.M);
	const MemberView& v = B.mv[sb.m];
	moments_prefix_body(GridSeg { sb.id, sb.n }, v.T, reinterpret_cast<const Mom5*>(v.T.mom_pre), nullptr, v.P,
	                    v.rec);
}

static_assert(MOM_TILE == (int)PACK_MOM_TILE, "moment tile");

void pack_keys(const PackDev& B, int k, cudaStream_t s)
{
	kp_keys<<<B.blocks[PS_KEYS], 256, 0, s>>>(B, k);
}

void pack_reorder(const PackDev& B, int k, cudaStream_t s)
{
	kp_reorder<<<B.blocks[PS_N256], 256, 0, s>>>(B, k);
}

// Octree and fast-form moments of every member (launch_build's sequence).
void pack_build(const PackDev& B, cudaStream_t s)
{
	kp_pairs<<<B.blocks[PS_PAIRS], 256, 0, s>>>(B);
	pack_node_scan(B, s);
	kp_fill_nodes<<<B.blocks[PS_FILL], 256, 0, s>>>(B);
	kp_finish_nodes<<<B.blocks[PS_FINISH], 256, 0, s>>>(B);
	kp_mom_reduce<<<B.blocks[PS_MOM], MOM_THREADS, 0, s>>>(B);
	kp_mom_top<<<B.blocks[PS_ONE], MOM_THREADS, 0, s>>>(B);
	kp_mom_down<<<B.blocks[PS_MOM], MOM_THREADS, 0, s>>>(B);
	kp_moments_prefix<<<B.blocks[PS_MOMPRE], 256, 0, s>>>(B);
}

}  // namespace pot
