// Fast form (POT_FORM_FAST): leaf-grouped, warp-cooperative Barnes-Hut walk
// in FP32, fused with the FP64 Boris push, absorption and boundary test.
//
// A warp owns a group of 32 consecutive due particles in Morton order (one
// per lane) and walks the tree once for the whole group:
//   * opening test per cell against the group's bounding box: accept when
//     the squared distance from the box to the cell's centre of charge
//     exceeds (x2 - x1)^2 / OAP^2.  Every target in the box is at least that
//     far, so each accepted cell also passes the reference's per-target test
//     (pot.c:1729); the group list refines every member's list;
//   * accepted cells (monopoles, unsoftened as pot.c:1737-1749) and opened
//     leaves (particle ranges, Plummer-softened as pot.c:1789-1798, the
//     target excluded by slot) are staged in shared memory and flushed:
//     every lane evaluates its own target against each staged entry, which
//     all lanes read at once;
//   * the stack of cells still to test lives in shared memory; children of
//     opened cells are appended with a warp prefix sum.
// Positions are FP32 relative to the domain centre in units of the domain
// radius; the FP32 sum is scaled to V/m in FP64 once per target.
#include "pot_push.cuh"

namespace pot {

constexpr int FW_WARPS = 4;        // warps per block
constexpr int FW_STACK = 1536;     // cells awaiting a test, per warp
constexpr int FW_CELLS = 96;       // staged monopoles (flush at >= 64)
constexpr int FW_CELL_FLUSH = 64;
constexpr int FW_LEAVES = 64;      // staged leaf ranges (flush at >= 32)
constexpr int FW_LEAF_FLUSH = 32;

struct FastSmem {
	int32_t stack[FW_STACK];
	float4 cells[FW_CELLS];
	uint2 leaves[FW_LEAVES];
	uint32_t loff[FW_LEAVES];  // exclusive prefix of the staged leaves' particle counts
	float4 pbuf[32];           // one 32-particle chunk of opened leaves
	uint32_t pidx[32];         // their slots (self exclusion)
};

__device__ __forceinline__ uint32_t lane_f() { return threadIdx.x & 31u; }

__device__ __forceinline__ float box_d2(float3 bmin, float3 bmax, float4 c)
{
	const float dx = fmaxf(fmaxf(bmin.x - c.x, c.x - bmax.x), 0.0f);
	const float dy = fmaxf(fmaxf(bmin.y - c.y, c.y - bmax.y), 0.0f);
	const float dz = fmaxf(fmaxf(bmin.z - c.z, c.z - bmax.z), 0.0f);
	return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ int warp_excl(int v, int& total)
{
	int incl = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int t = __shfl_up_sync(0xffffffffu, incl, o);
		if ((int)lane_f() >= o) incl += t;
	}
	total = __shfl_sync(0xffffffffu, incl, 31);
	return incl - v;
}

// Group walk.  t = target (relative units), self = own slot (or 0xFFFFFFFF),
// valid = lane holds a target.  Returns E in units of q / R^2 (multiply by
// QE / (4 pi eps0 R^2) for V/m) and the number of entries evaluated.
__device__ float3 group_walk(float3 t, uint32_t self, bool valid, const TreeDev& T,
                             const float4* __restrict__ src32, const Params& P, FastSmem& sm,
                             uint32_t& n_eval, int& err)
{
	const uint32_t lane = lane_f();
	// group bounding box over valid lanes
	const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
	const int src_lane = vmask ? __ffs(vmask) - 1 : 0;
	float3 ref = make_float3(__shfl_sync(0xffffffffu, t.x, src_lane), __shfl_sync(0xffffffffu, t.y, src_lane),
	                         __shfl_sync(0xffffffffu, t.z, src_lane));
	float3 q = valid ? t : ref;
	float3 bmin = q, bmax = q;
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		bmin.x = fminf(bmin.x, __shfl_xor_sync(0xffffffffu, bmin.x, o));
		bmin.y = fminf(bmin.y, __shfl_xor_sync(0xffffffffu, bmin.y, o));
		bmin.z = fminf(bmin.z, __shfl_xor_sync(0xffffffffu, bmin.z, o));
		bmax.x = fmaxf(bmax.x, __shfl_xor_sync(0xffffffffu, bmax.x, o));
		bmax.y = fmaxf(bmax.y, __shfl_xor_sync(0xffffffffu, bmax.y, o));
		bmax.z = fmaxf(bmax.z, __shfl_xor_sync(0xffffffffu, bmax.z, o));
	}
	const float eps2 = P.soft2_f;
	const bool single_leaves = P.leaf_size == 1;
	float ex = 0.f, ey = 0.f, ez = 0.f;
	int len = 1, ncell = 0, nleaf = 0;
	uint32_t n_cells_ev = 0, n_parts_ev = 0;
	if (lane == 0) sm.stack[0] = 0;
	__syncwarp();
	for (;;) {
		const bool done = (len == 0);
		if (!done) {
			const int take = len < 32 ? len : 32;
			const int32_t code = (int)lane < take ? sm.stack[len - 1 - (int)lane] : CH_EMPTY;
			__syncwarp();
			len -= take;
			bool acc = false, leafr = false;
			float4 cell = make_float4(0.f, 0.f, 0.f, 0.f);
			uint2 range = make_uint2(0u, 0u);
			int nch = 0;
			int32_t ch[8];
			if (code >= 0) {
				cell = T.f[code];
				if (box_d2(bmin, bmax, cell) > T.r2[code]) {
					acc = cell.w != 0.f;
				} else {
					const int4* cp = reinterpret_cast<const int4*>(&T.child[8u * (uint32_t)code]);
					const int4 c0 = cp[0], c1 = cp[1];
					const int32_t cc[8] = { c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w };
#pragma unroll
					for (int d = 0; d < 8; d++)
						if (cc[d] != CH_EMPTY) ch[nch++] = cc[d];
				}
			} else if (code != CH_EMPTY) {
				const uint32_t e = leaf_payload(code);
				if (single_leaves) {
					leafr = true;
					range = e < P.n ? make_uint2(e, 1u) : T.ovf[e - P.n];
				} else {
					cell = T.lf[e];
					if (box_d2(bmin, bmax, cell) > T.lr2[e]) {
						acc = cell.w != 0.f;
					} else {
						leafr = true;
						range = T.lrange[e];
					}
				}
			}
			int tot;
			const int co = warp_excl(acc ? 1 : 0, tot);
			if (acc) sm.cells[ncell + co] = cell;
			ncell += tot;
			const int lo = warp_excl(leafr ? 1 : 0, tot);
			if (leafr) sm.leaves[nleaf + lo] = range;
			nleaf += tot;
			const int po = warp_excl(nch, tot);
			if (len + tot > FW_STACK) {
				err = POT_E_WALK;
				break;
			}
			for (int j = 0; j < nch; j++) sm.stack[len + po + j] = ch[j];
			len += tot;
			__syncwarp();
		}
		// flush staged monopoles
		if (ncell >= FW_CELL_FLUSH || (done && ncell > 0)) {
#pragma unroll 4
			for (int j = 0; j < ncell; j++) {
				const float4 c = sm.cells[j];
				const float dx = t.x - c.x, dy = t.y - c.y, dz = t.z - c.z;
				const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
				const float ri = rsqrtf(r2);
				const float w = c.w * ri * ri * ri;
				ex = fmaf(w, dx, ex);
				ey = fmaf(w, dy, ey);
				ez = fmaf(w, dz, ez);
			}
			n_cells_ev += ncell;
			ncell = 0;
			__syncwarp();
		}
		// flush staged leaves: their particles are gathered 32 at a time into
		// shared memory (dense, by a prefix sum over the leaf sizes) and every
		// lane evaluates its target against each of them
		if (nleaf >= FW_LEAF_FLUSH || (done && nleaf > 0)) {
			const uint32_t c0 = (int)lane < nleaf ? sm.leaves[lane].y : 0u;
			const uint32_t c1 = (int)lane + 32 < nleaf ? sm.leaves[lane + 32].y : 0u;
			int t0, t1;
			const int e0 = warp_excl((int)c0, t0);
			const int e1 = warp_excl((int)c1, t1);
			sm.loff[lane] = (uint32_t)e0;
			sm.loff[lane + 32] = (uint32_t)(t0 + e1);
			const uint32_t total = (uint32_t)(t0 + t1);
			__syncwarp();
			for (uint32_t base = 0; base < total; base += 32) {
				const uint32_t g = base + lane;
				float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
				uint32_t id = 0xFFFFFFFFu;
				if (g < total) {
					int lo = 0, hi = nleaf - 1;
					while (lo < hi) {  // last staged leaf whose offset <= g
						const int mid = (lo + hi + 1) >> 1;
						if (sm.loff[mid] <= g) lo = mid; else hi = mid - 1;
					}
					id = sm.leaves[lo].x + (g - sm.loff[lo]);
					p = __ldg(&src32[id]);
				}
				sm.pbuf[lane] = p;
				sm.pidx[lane] = id;
				__syncwarp();
#pragma unroll 8
				for (int m = 0; m < 32; m++) {
					const float4 q = sm.pbuf[m];
					const float dx = t.x - q.x, dy = t.y - q.y, dz = t.z - q.z;
					const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
					const float ri = rsqrtf(r2);
					const float w = (sm.pidx[m] == self) ? 0.f : q.w * ri * ri * ri;
					ex = fmaf(w, dx, ex);
					ey = fmaf(w, dy, ey);
					ez = fmaf(w, dz, ez);
				}
				__syncwarp();
			}
			n_parts_ev += total;
			nleaf = 0;
			__syncwarp();
		}
		if (done) break;
	}
	n_eval = valid ? n_cells_ev + n_parts_ev : 0u;
	return make_float3(ex, ey, ez);
}

// Slot range [a, b) of a child code.
__device__ __forceinline__ void child_range(const TreeDev& T, int32_t code, const Params& P, uint32_t& a, uint32_t& b)
{
	if (code >= 0) {
		a = T.first[code];
		b = T.last[code] + 1;
		return;
	}
	const uint32_t e = leaf_payload(code);
	if (P.leaf_size == 1) {
		if (e < P.n) {
			a = e;
			b = e + 1;
		} else {
			const uint2 r = T.ovf[e - P.n];
			a = r.x;
			b = r.x + r.y;
		}
	} else {
		const uint2 r = T.lrange[e];
		a = r.x;
		b = r.x + r.y;
	}
}

__device__ __forceinline__ void emit_groups(RunRec* rec, uint2* groups, uint32_t start, uint32_t count)
{
	while (count > 0) {
		const uint32_t c = count < GROUP_MAX ? count : GROUP_MAX;
		groups[atomicAdd(&rec->n_groups, 1u)] = make_uint2(start, c);
		start += c;
		count -= c;
	}
}

// Target groups aligned with tree cells.  dpre[s] = due particles in slots
// [0, s).  A cell with more than GROUP_MAX due particles packs its children,
// in key order, into runs of at most GROUP_MAX due particles (children with
// more start their own packing); so every group lies inside one parent cell
// and its bounding box stays compact.  A group is a range of the due list.
__global__ void k_groups(TreeDev T, const uint32_t* __restrict__ dpre, uint2* __restrict__ groups, Params P,
                         RunRec* rec)
{
	if (rec->status != POT_OK) return;
	const uint32_t M = rec->n_nodes;
	for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
		const uint32_t a = T.first[k], b = T.last[k] + 1;
		const uint32_t d = dpre[b] - dpre[a];
		if (d == 0) continue;
		if (d <= GROUP_MAX) {
			if (k == 0) emit_groups(rec, groups, dpre[a], d);
			continue;
		}
		uint32_t run_start = 0, run = 0;
		for (int c = 0; c < 8; c++) {
			const int32_t code = T.child[8u * k + (uint32_t)c];
			if (code == CH_EMPTY) continue;
			uint32_t ca, cb;
			child_range(T, code, P, ca, cb);
			const uint32_t dc = dpre[cb] - dpre[ca];
			if (dc == 0) continue;
			if (code >= 0 && dc > GROUP_MAX) {
				emit_groups(rec, groups, run_start, run);
				run = 0;
				continue;
			}
			if (run + dc > GROUP_MAX) {
				emit_groups(rec, groups, run_start, run);
				run = 0;
			}
			if (run == 0) run_start = dpre[ca];
			run += dc;
		}
		emit_groups(rec, groups, run_start, run);
	}
}

__global__ void __launch_bounds__(FW_WARPS * 32) k_push_fast(double4* __restrict__ pos, double4* __restrict__ vel,
                                                            TreeDev T, const float4* __restrict__ src32,
                                                            const uint32_t* __restrict__ due_list,
                                                            const uint2* __restrict__ groups,
                                                            uint32_t* __restrict__ rein_list, Params P,
                                                            RunRec* rec)
{
	__shared__ FastSmem smem[FW_WARPS];
	FastSmem& sm = smem[threadIdx.x >> 5];
	if (rec->status != POT_OK) return;
	const uint32_t n_groups = rec->n_groups;
	const unsigned long long t_step = rec->t_steps;
	const bool grain_due = rec->grain_due != 0;
	const bool absorb_on = !(P.flags & FLAG_NO_GRAIN) && t_step >= P.t_settle;
	const double gx = rec->grain_pos[0], gy = rec->grain_pos[1], gz = rec->grain_pos[2];
	const double qg = (double)rec->grain_q;
	const double escale = QE / (P.k4 * P.rad * P.rad);
	unsigned long long n_inter = 0, n_push = 0;
	for (;;) {
		uint32_t g = 0;
		if (lane_f() == 0) g = atomicAdd(&rec->work_ctr, 1u);
		g = __shfl_sync(0xffffffffu, g, 0);
		if (g >= n_groups) break;
		const uint2 grp = groups[g];
		const uint32_t i = grp.x + lane_f();
		const bool valid = lane_f() < grp.y;
		uint32_t s = 0xFFFFFFFFu;
		double4 p = make_double4(P.rad, P.rad, P.rad, 0.0), v = make_double4(0.0, 0.0, 0.0, 0.0);
		int sp = SP_E;
		double dt = P.dt, half = 0.5 * P.dt;
		double3 h = make_double3(P.rad, P.rad, P.rad);
		if (valid) {
			s = due_list[i];
			p = pos[s];
			v = vel[s];
			sp = (int)p.w;
			dt = P.dt * (double)P.tss[sp];
			half = 0.5 * dt;
			h = make_double3(fma(half, v.x, p.x), fma(half, v.y, p.y), fma(half, v.z, p.z));
		}
		const float3 tf = make_float3((float)((h.x - P.rad) * P.inv_rad), (float)((h.y - P.rad) * P.inv_rad),
		                              (float)((h.z - P.rad) * P.inv_rad));
		uint32_t ne = 0;
		int err = POT_OK;
		const float3 ef = group_walk(tf, s, valid, T, src32, P, sm, ne, err);
		if (err != POT_OK) {
			if (lane_f() == 0) set_status(rec, err);
			break;
		}
		if (!valid) continue;
		n_inter += ne;
		n_push++;
		const double E[3] = { (double)ef.x * escale, (double)ef.y * escale, (double)ef.z * escale };
		const double charge = sp == SP_DUST ? qg : (sp == SP_ION ? 1.0 : -1.0);
		const double mass = sp == SP_DUST ? MASS_DUST : (sp == SP_ION ? MASS_ION : MASS_E);
		const double qom = (QE * charge) / mass;
		double3 xn;
		boris(v, h, E, qom, dt, P, xn);
		uint32_t reason = 0;
		if (!grain_due) reason = after_push(sp, p, xn, v, P, rec, absorb_on, gx, gy, gz);
		pos[s] = make_double4(xn.x, xn.y, xn.z, p.w);
		vel[s] = v;
		if (reason) rein_list[atomicAdd(&rec->n_rein, 1u)] = s | (reason << 30);
	}
	unsigned long long a = n_inter, b = n_push;
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		a += __shfl_xor_sync(0xffffffffu, a, o);
		b += __shfl_xor_sync(0xffffffffu, b, o);
	}
	if (lane_f() == 0) {
		if (a) atomicAdd(&rec->interactions, a);
		if (b) atomicAdd(&rec->n_pushed, b);
	}
}

__global__ void __launch_bounds__(FW_WARPS * 32) k_field_query_fast(TreeDev T, const float4* __restrict__ src32,
                                                                   const double* __restrict__ xyz,
                                                                   const uint32_t* __restrict__ self_slot,
                                                                   uint32_t nq, double* __restrict__ E, Params P,
                                                                   RunRec* rec)
{
	__shared__ FastSmem smem[FW_WARPS];
	FastSmem& sm = smem[threadIdx.x >> 5];
	const uint32_t n_groups = (nq + 31) / 32;
	const double escale = QE / (P.k4 * P.rad * P.rad);
	for (uint32_t g = blockIdx.x * FW_WARPS + (threadIdx.x >> 5); g < n_groups; g += gridDim.x * FW_WARPS) {
		const uint32_t q = g * 32 + lane_f();
		const bool valid = q < nq;
		float3 tf = make_float3(0.f, 0.f, 0.f);
		uint32_t self = 0xFFFFFFFFu;
		if (valid) {
			tf = make_float3((float)((xyz[3 * q] - P.rad) * P.inv_rad), (float)((xyz[3 * q + 1] - P.rad) * P.inv_rad),
			                 (float)((xyz[3 * q + 2] - P.rad) * P.inv_rad));
			self = self_slot[q];
		}
		uint32_t ne = 0;
		int err = POT_OK;
		const float3 ef = group_walk(tf, self, valid, T, src32, P, sm, ne, err);
		if (err != POT_OK && lane_f() == 0) set_status(rec, err);
		if (valid) {
			E[3 * q] = (double)ef.x * escale;
			E[3 * q + 1] = (double)ef.y * escale;
			E[3 * q + 2] = (double)ef.z * escale;
		}
	}
}

static int sm_count_fast()
{
	static int n = 0;
	if (!n) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		if (n <= 0) n = 148;
	}
	return n;
}

void launch_groups(const TreeDev& T, const uint32_t* dpre, uint2* groups, const Params& P, RunRec* rec,
                   cudaStream_t s, Timer& tm)
{
	cudaMemsetAsync(&rec->n_groups, 0, sizeof(unsigned int), s);
	ScopedKernel k(tm, "groups");
	k_groups<<<sm_count_fast() * 4, 256, 0, s>>>(T, dpre, groups, P, rec);
}

void launch_push_fast(double4* pos, double4* vel, const TreeDev& T, const float4* src32, const double4* src64,
                      const uint32_t* due_list, const uint2* groups, uint32_t* rein_list, const Params& P,
                      RunRec* rec, cudaStream_t s, Timer& tm)
{
	(void)src64;
	ScopedKernel k(tm, "walk_push_fast");
	k_push_fast<<<sm_count_fast() * 6, FW_WARPS * 32, 0, s>>>(pos, vel, T, src32, due_list, groups, rein_list, P,
	                                                         rec);
}

void launch_field_query_fast(const TreeDev& T, const float4* src32, const double* xyz, const uint32_t* self_slot,
                             uint32_t nq, double* E, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "field_query_fast");
	const uint32_t groups = (nq + 31) / 32;
	uint32_t nb = (groups + FW_WARPS - 1) / FW_WARPS;
	if (nb == 0) nb = 1;
	k_field_query_fast<<<nb, FW_WARPS * 32, 0, s>>>(T, src32, xyz, self_slot, nq, E, P, rec);
}

}  // namespace pot
