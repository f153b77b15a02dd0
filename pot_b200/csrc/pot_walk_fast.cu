// Fast form (POT_FORM_FAST): leaf-grouped, warp-cooperative Barnes-Hut walk
// in FP32, fused with the FP64 Boris push, absorption and boundary test.
//
// Groups.  Targets are the particles due this step, in Morton order.  A group
// is a run of at most GROUP_MAX (64) of them lying inside one tree cell (see
// k_groups), so its bounding box is compact.  A warp owns one group, one or
// two targets per lane.
//
// Walk.  The warp walks the tree once for the whole group:
//   * opening test per cell: the reference's test (pot.c:1729), accept when
//     (x2 - x1)^2 < OAP^2 d^2, with d the distance from the centre of the
//     group's bounding box to the cell's centre of charge -- the test of the
//     group's typical member -- and only if no member can lie inside the
//     cell: the box must be farther from the centre of charge than the
//     cell's diagonal, sqrt(3) (x2 - x1), so a cell never holds a target it
//     is accepted for (the reference's self-inclusion at OAP >= 1/sqrt(3)
//     does not occur);
//   * accepted cells (monopoles, unsoftened as pot.c:1737-1749) are staged in
//     shared memory; opened leaves (particle ranges, Plummer-softened as
//     pot.c:1789-1798, the target excluded by slot) are staged as ranges and
//     their particles gathered 32 at a time into shared memory;
//   * flushes: every lane evaluates its two targets against each staged
//     entry, which all lanes read at once (shared-memory broadcast);
//   * the stack of cells still to test lives in shared memory; children of
//     opened cells are appended with a warp prefix sum.
// Positions are FP32 relative to the domain centre in units of the domain
// radius; the FP32 sums are scaled to V/m in FP64 once per target.
#include "pot_push.cuh"

namespace pot {

constexpr int FW_WARPS = 4;        // warps per block
constexpr int FW_TPL_MAX = 2;      // targets per lane (1 or 2; groups of 32 or 64)
constexpr int FW_STACK = POT_WALK_STACK;  // cells awaiting a test, per warp
constexpr int FW_CELLS = 104;      // staged monopoles (flush at >= 64; at most 95 staged, 96 padded)
constexpr int FW_CELL_FLUSH = 64;
constexpr int FW_LEAVES = 64;      // staged leaf ranges (flush at >= 32)
constexpr int FW_LEAF_FLUSH = 32;
static_assert(GROUP_MAX == 32 * FW_TPL_MAX, "one group per warp, at most FW_TPL_MAX targets per lane");
// Blocks per SM the push kernels are compiled for.  With two targets per
// lane the walk holds both targets' sums and operands: at four blocks (128
// registers a thread) it needs no spills and runs faster than at five (96
// registers, spilling), 4.51 against 4.65 ms per step on the 4m plasma.  One
// target per lane fits 96 registers, and five blocks hide more latency.
constexpr int fw_push_blocks(int tpl) { return tpl == 2 ? 4 : 5; }

// Per-warp shared memory.  A staged source (accepted cell or gathered
// particle) takes TPL float4s: with one target per lane it is (x, y, z, q);
// with two it is stored duplicated and negated as (-x, -x, -y, -y),
// (-z, -z, q, q) so that each half is a ready operand of the packed FP32x2
// instructions that evaluate both targets of a lane at once.
// With DIPOLES (one target per lane) the cell buffer has a second half that
// holds each staged cell's dipole moment, packed in pairs like the positions.
template <int TPL, bool DIP = false>
struct FastSmem {
	int32_t stack[FW_STACK];
	float4 cells[FW_CELLS * TPL * (DIP ? 2 : 1)];
	uint2 leaves[FW_LEAVES];
	uint32_t loff[FW_LEAVES];  // exclusive prefix of the staged leaves' particle counts
	float4 pbuf[32 * TPL];     // one 32-particle chunk of opened leaves
};

__device__ __forceinline__ uint32_t lane_f() { return threadIdx.x & 31u; }

__device__ __forceinline__ float box_d2(float3 bmin, float3 bmax, float4 c)
{
	const float dx = fmaxf(fmaxf(bmin.x - c.x, c.x - bmax.x), 0.0f);
	const float dy = fmaxf(fmaxf(bmin.y - c.y, c.y - bmax.y), 0.0f);
	const float dz = fmaxf(fmaxf(bmin.z - c.z, c.z - bmax.z), 0.0f);
	return dx * dx + dy * dy + dz * dz;
}

// The group's opening test (see the file comment).  r2 = (x2 - x1)^2 / OAP^2
// in units of R^2, th2 = OAP^2; bc the centre of the group's box.
__device__ __forceinline__ bool group_accepts(float3 bmin, float3 bmax, float3 bc, float4 c, float r2, float th2)
{
	const float db2 = box_d2(bmin, bmax, c);
	if (db2 <= 3.0f * th2 * r2) return false;  // a member may lie inside the cell
	const float dx = bc.x - c.x, dy = bc.y - c.y, dz = bc.z - c.z;
	return dx * dx + dy * dy + dz * dz > r2;
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

template <int TPL>
struct Targets {
	float3 t[TPL];
	uint32_t self[TPL];  // slot, 0xFFFFFFFF for none
	bool valid[TPL];
};

template <int TPL>
struct Field {
	float x[TPL], y[TPL], z[TPL];
};

// Field sums in evaluation form: scalars for one target per lane; for two,
// FP32x2 pairs (target 0 in .x, target 1 in .y).
template <int TPL> struct Acc;
template <> struct Acc<1> { float x, y, z; };
template <> struct Acc<2> { float2 x, y, z; };

template <int TPL> struct TgtE;
template <> struct TgtE<1> { float x, y, z; };
template <> struct TgtE<2> { float2 x, y, z; };

// FP32 reciprocal square root: the hardware approximation with subnormal
// input flushed to zero (PTX rsqrt.approx.ftz.f32), one instruction.  Its
// arguments are squared distances to accepted cells or softened (floor
// 1e-20 R^2) squared distances to particles, never subnormal, where the
// flushing and the non-flushing forms give the same result.
__device__ __forceinline__ float rsqrt_ftz(float x)
{
	float r;
	asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
}

__device__ __forceinline__ void stage_src(float4* buf, int i, float4 c, Acc<1>*) { buf[i] = c; }
__device__ __forceinline__ void stage_src(float4* buf, int i, float4 c, Acc<2>*)
{
	buf[2 * i] = make_float4(-c.x, -c.x, -c.y, -c.y);
	buf[2 * i + 1] = make_float4(-c.z, -c.z, c.w, c.w);
}

// One source against the lane's target(s).  SOFT: Plummer-softened pair
// (pot.c:1789-1798); else an unsoftened monopole (pot.c:1737-1749).  POT:
// accumulate q / r in .x (pot.c:1960-1973).  The operation order is the same
// in both forms: r2 = dx dx + (dy dy + (dz dz [+ eps2])), w = (q ri^2) ri.
template <bool SOFT, bool POT>
__device__ __forceinline__ void eval_src(Acc<1>& E, const TgtE<1>& t, const float4* buf, int i, float eps2)
{
	const float4 q = buf[i];
	const float dx = t.x - q.x, dy = t.y - q.y, dz = t.z - q.z;
	const float r2 = fmaf(dx, dx, fmaf(dy, dy, SOFT ? fmaf(dz, dz, eps2) : dz * dz));
	const float ri = rsqrt_ftz(r2);
	if (POT) {
		E.x = fmaf(q.w, ri, E.x);
	} else {
		const float w = q.w * (ri * ri) * ri;
		E.x = fmaf(w, dx, E.x);
		E.y = fmaf(w, dy, E.y);
		E.z = fmaf(w, dz, E.z);
	}
}

template <bool SOFT, bool POT>
__device__ __forceinline__ void eval_src(Acc<2>& E, const TgtE<2>& t, const float4* buf, int i, float eps2)
{
	const float4 a = buf[2 * i], b = buf[2 * i + 1];
	const float2 dx = __fadd2_rn(t.x, make_float2(a.x, a.y));
	const float2 dy = __fadd2_rn(t.y, make_float2(a.z, a.w));
	const float2 dz = __fadd2_rn(t.z, make_float2(b.x, b.y));
	const float2 q = make_float2(b.z, b.w);
	float2 r2 = SOFT ? __ffma2_rn(dz, dz, make_float2(eps2, eps2)) : __fmul2_rn(dz, dz);
	r2 = __ffma2_rn(dy, dy, r2);
	r2 = __ffma2_rn(dx, dx, r2);
	const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
	if (POT) {
		E.x = __ffma2_rn(q, ri, E.x);
	} else {
		const float2 w = __fmul2_rn(__fmul2_rn(q, __fmul2_rn(ri, ri)), ri);
		E.x = __ffma2_rn(w, dx, E.x);
		E.y = __ffma2_rn(w, dy, E.y);
		E.z = __ffma2_rn(w, dz, E.z);
	}
}

// Two staged sources (x, y, z, q) in float4 slots 2p and 2p + 1 become one
// FP32x2 operand pair, (-xa, -xb, -ya, -yb) and (-za, -zb, qa, qb), in place:
// with one target per lane the packed instructions evaluate two sources at
// once against the (duplicated) target.
__device__ __forceinline__ void pair_pack(float4* buf, int p)
{
	const float4 a = buf[2 * p], b = buf[2 * p + 1];
	buf[2 * p] = make_float4(-a.x, -b.x, -a.y, -b.y);
	buf[2 * p + 1] = make_float4(-a.z, -b.z, a.w, b.w);
}

// the dipoles of two staged cells, (px, py, pz, 0) in slots 2p and 2p + 1,
// become (pxa, pxb, pya, pyb), (pza, pzb, 0, 0), in place
__device__ __forceinline__ void pair_pack_dip(float4* buf, int p)
{
	const float4 a = buf[2 * p], b = buf[2 * p + 1];
	buf[2 * p] = make_float4(a.x, b.x, a.y, b.y);
	buf[2 * p + 1] = make_float4(a.z, b.z, 0.f, 0.f);
}

// Two staged cells with their dipoles (DIPOLES, pot.c:1739-1745) against the
// duplicated target: E += (q + 3 (p.r) / r^2) r / r^3 - p / r^3, or for the
// potential q / r + (p.r) / r^3 (pot.c:1966-1974), r from the cell's centre
// of charge to the target; cells unsoftened.
template <bool POT>
__device__ __forceinline__ void eval_cell_dip(Acc<2>& E, const TgtE<2>& t, const float4* buf, const float4* dbuf,
                                              int i)
{
	const float4 a = buf[2 * i], b = buf[2 * i + 1], pa = dbuf[2 * i], pb = dbuf[2 * i + 1];
	const float2 dx = __fadd2_rn(t.x, make_float2(a.x, a.y));
	const float2 dy = __fadd2_rn(t.y, make_float2(a.z, a.w));
	const float2 dz = __fadd2_rn(t.z, make_float2(b.x, b.y));
	const float2 q = make_float2(b.z, b.w);
	const float2 px = make_float2(pa.x, pa.y), py = make_float2(pa.z, pa.w), pz = make_float2(pb.x, pb.y);
	float2 r2 = __fmul2_rn(dz, dz);
	r2 = __ffma2_rn(dy, dy, r2);
	r2 = __ffma2_rn(dx, dx, r2);
	const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
	const float2 ri2 = __fmul2_rn(ri, ri);
	const float2 ri3 = __fmul2_rn(ri2, ri);
	float2 pr = __fmul2_rn(pz, dz);
	pr = __ffma2_rn(py, dy, pr);
	pr = __ffma2_rn(px, dx, pr);
	if (POT) {
		E.x = __ffma2_rn(q, ri, E.x);
		E.x = __ffma2_rn(pr, ri3, E.x);
	} else {
		const float2 w = __fmul2_rn(ri3, __ffma2_rn(make_float2(3.f, 3.f), __fmul2_rn(pr, ri2), q));
		const float2 nri3 = make_float2(-ri3.x, -ri3.y);
		E.x = __ffma2_rn(nri3, px, __ffma2_rn(w, dx, E.x));
		E.y = __ffma2_rn(nri3, py, __ffma2_rn(w, dy, E.y));
		E.z = __ffma2_rn(nri3, pz, __ffma2_rn(w, dz, E.z));
	}
}

__device__ __forceinline__ void add_xor(Acc<1>& E, int o)
{
	E.x += __shfl_xor_sync(0xffffffffu, E.x, o);
	E.y += __shfl_xor_sync(0xffffffffu, E.y, o);
	E.z += __shfl_xor_sync(0xffffffffu, E.z, o);
}
__device__ __forceinline__ void add_xor(Acc<2>& E, int o)
{
	E.x.x += __shfl_xor_sync(0xffffffffu, E.x.x, o);
	E.x.y += __shfl_xor_sync(0xffffffffu, E.x.y, o);
	E.y.x += __shfl_xor_sync(0xffffffffu, E.y.x, o);
	E.y.y += __shfl_xor_sync(0xffffffffu, E.y.y, o);
	E.z.x += __shfl_xor_sync(0xffffffffu, E.z.x, o);
	E.z.y += __shfl_xor_sync(0xffffffffu, E.z.y, o);
}

__device__ __forceinline__ void to_eval(const Targets<1>& tg, TgtE<1>& t, Acc<1>& E)
{
	t.x = tg.t[0].x;
	t.y = tg.t[0].y;
	t.z = tg.t[0].z;
	E.x = E.y = E.z = 0.f;
}
__device__ __forceinline__ void to_eval(const Targets<2>& tg, TgtE<2>& t, Acc<2>& E)
{
	t.x = make_float2(tg.t[0].x, tg.t[1].x);
	t.y = make_float2(tg.t[0].y, tg.t[1].y);
	t.z = make_float2(tg.t[0].z, tg.t[1].z);
	E.x = E.y = E.z = make_float2(0.f, 0.f);
}
__device__ __forceinline__ Field<1> from_eval(const Acc<1>& E)
{
	Field<1> f;
	f.x[0] = E.x;
	f.y[0] = E.y;
	f.z[0] = E.z;
	return f;
}
__device__ __forceinline__ Field<2> from_eval(const Acc<2>& E)
{
	Field<2> f;
	f.x[0] = E.x.x;
	f.x[1] = E.x.y;
	f.y[0] = E.y.x;
	f.y[1] = E.y.y;
	f.z[0] = E.z.x;
	f.z[1] = E.z.y;
	return f;
}

// Far cells of a group.  An accepted cell whose centre of charge is farther
// from the centre c of the group's box than FAR_RATIO times h, the largest
// distance of a member from c, is not staged for every target: the lane
// that tested it adds
// its field at c and the field's first and second derivatives there to the
// lane's expansion (monopole field E = q d / r^3, d = t - s):
//   E_a     = w d_a,                                  w = q / r^3
//   J_ab    = w (delta_ab - 3 d_a d_b / r^2)          (symmetric, traceless)
//   H_abc   = w / r^2 (15 d_a d_b d_c / r^2 - 3 (delta_ab d_c + delta_ac d_b
//             + delta_bc d_a))                        (symmetric, traceless)
// J keeps 5 components, H 7 (J_zz = -J_xx - J_yy, H_xzz = -H_xxx - H_xyy,
// H_yzz = -H_xxy - H_yyy, H_zzz = -H_xxz - H_yyz: a monopole's field is
// divergence-free away from it).  After the walk the lanes' expansions are
// summed by shuffles and each target adds E + J delta + H delta delta / 2,
// delta = t - c.  The remainder is of third order: with e = |delta| / d <=
// 1 / FAR_RATIO it is at most 1 / (1 - e)^2 - (1 + 2 e + 3 e^2) of the
// cell's field at c (leading term 4 e^3; reached towards the cell), 9.0 %
// for a ratio of 4, comparable to the monopole's own truncation of the
// cell's dipole and quadrupole, which the opening test bounds by theta.  On
// the 4m plasma ratios 4, 5 and 6 give the push the same field error against
// a direct sum (8.2 %, 8.3 % and 8.3 % RMS); 4 stages the fewest terms.
constexpr float FAR_RATIO = 4.0f;

struct FarExp {
	float ex, ey, ez;
	float jxx, jyy, jxy, jxz, jyz;
	float hxxx, hyyy, hxxy, hxxz, hxyy, hyyz, hxyz;
	__device__ __forceinline__ void zero()
	{
		ex = ey = ez = 0.f;
		jxx = jyy = jxy = jxz = jyz = 0.f;
		hxxx = hyyy = hxxy = hxxz = hxyy = hyyz = hxyz = 0.f;
	}
	// a monopole of charge q at (sx, sy, sz), expanded about c
	__device__ __forceinline__ void add(float3 c, float4 s)
	{
		const float dx = c.x - s.x, dy = c.y - s.y, dz = c.z - s.z;
		const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
		const float ri = rsqrt_ftz(r2);
		const float ri2 = ri * ri;
		const float w = (s.w * ri2) * ri;
		ex = fmaf(w, dx, ex);
		ey = fmaf(w, dy, ey);
		ez = fmaf(w, dz, ez);
		const float w3 = -3.f * w * ri2;  // -3 w / r^2
		jxx += fmaf(w3, dx * dx, w);
		jyy += fmaf(w3, dy * dy, w);
		jxy = fmaf(w3, dx * dy, jxy);
		jxz = fmaf(w3, dx * dz, jxz);
		jyz = fmaf(w3, dy * dz, jyz);
		// H_abc = v15 d_a d_b d_c + v3 (delta_ab d_c + delta_ac d_b + delta_bc d_a)
		const float v3 = w3;                // -3 w / r^2
		const float v15 = -5.f * w3 * ri2;  // 15 w / r^4
		hxxx += dx * fmaf(v15, dx * dx, 3.f * v3);
		hyyy += dy * fmaf(v15, dy * dy, 3.f * v3);
		hxxy += dy * fmaf(v15, dx * dx, v3);
		hxxz += dz * fmaf(v15, dx * dx, v3);
		hxyy += dx * fmaf(v15, dy * dy, v3);
		hyyz += dz * fmaf(v15, dy * dy, v3);
		hxyz = fmaf(v15 * dx, dy * dz, hxyz);
	}
	__device__ __forceinline__ void warp_sum()
	{
#pragma unroll
		for (int o = 16; o; o >>= 1) {
			ex += __shfl_xor_sync(0xffffffffu, ex, o);
			ey += __shfl_xor_sync(0xffffffffu, ey, o);
			ez += __shfl_xor_sync(0xffffffffu, ez, o);
			jxx += __shfl_xor_sync(0xffffffffu, jxx, o);
			jyy += __shfl_xor_sync(0xffffffffu, jyy, o);
			jxy += __shfl_xor_sync(0xffffffffu, jxy, o);
			jxz += __shfl_xor_sync(0xffffffffu, jxz, o);
			jyz += __shfl_xor_sync(0xffffffffu, jyz, o);
			hxxx += __shfl_xor_sync(0xffffffffu, hxxx, o);
			hyyy += __shfl_xor_sync(0xffffffffu, hyyy, o);
			hxxy += __shfl_xor_sync(0xffffffffu, hxxy, o);
			hxxz += __shfl_xor_sync(0xffffffffu, hxxz, o);
			hxyy += __shfl_xor_sync(0xffffffffu, hxyy, o);
			hyyz += __shfl_xor_sync(0xffffffffu, hyyz, o);
			hxyz += __shfl_xor_sync(0xffffffffu, hxyz, o);
		}
	}
	// the expansion's field at c + (x, y, z)
	__device__ __forceinline__ float3 at(float x, float y, float z) const
	{
		const float jzz = -jxx - jyy;
		const float hxzz = -hxxx - hxyy, hyzz = -hxxy - hyyy, hzzz = -hxxz - hyyz;
		const float xx = 0.5f * x * x, yy = 0.5f * y * y, zz = 0.5f * z * z, xy = x * y, xz = x * z, yz = y * z;
		float3 e;
		e.x = ex + jxx * x + jxy * y + jxz * z + hxxx * xx + hxyy * yy + hxzz * zz + hxxy * xy + hxxz * xz + hxyz * yz;
		e.y = ey + jxy * x + jyy * y + jyz * z + hxxy * xx + hyyy * yy + hyzz * zz + hxyy * xy + hxyz * xz + hyyz * yz;
		e.z = ez + jxz * x + jyz * y + jzz * z + hxxz * xx + hyyz * yy + hzzz * zz + hxyz * xy + hxzz * xz + hyzz * yz;
		return e;
	}
};

// Group walk.  Returns the fields in units of q / R^2 (multiply by
// QE / (4 pi eps0 R^2) for V/m) and the number of entries evaluated per
// target.
//
// Self exclusion (pot.c:1789, node->part != part).  A target's own particle
// can only be evaluated as a particle of an opened leaf.  Opened leaves
// whose slot range meets the group's [min, max] self slots are few (the
// group lies inside one cell); for those the lanes test membership, and a
// target whose own particle was evaluated gets that same FP32 term
// subtracted at the end.  The softening is floored at 1e-20 R^2 (far below
// FP32 resolution of positions) so that the term is finite when a target sits
// exactly on its own particle.
//
// Split lists (one target per lane).  A group of at most 16 (8) targets
// would leave half (three quarters) of the warp idle during evaluation, so
// the lanes are split instead: lane l holds member l mod 32/split and
// evaluates the staged entries with index = sub (mod split), sub = l div
// 32/split; the split partial fields are added across lanes at the end.
template <int TPL, bool POT = false, bool DIP = false>
__device__ Field<TPL> group_walk(const Targets<TPL>& tg, const TreeDev& T, const float4* __restrict__ src32,
                                 const Params& P, FastSmem<TPL, DIP>& sm, uint32_t& n_eval, uint32_t& stack_max,
                                 int& err, int split = 1, uint32_t* n_far_cells = nullptr)
{
	const uint32_t lane = lane_f();
	uint32_t smin = 0xFFFFFFFFu, smax = 0u;
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		if (tg.valid[k] && tg.self[k] != 0xFFFFFFFFu) {
			smin = min(smin, tg.self[k]);
			smax = max(smax, tg.self[k]);
		}
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		smin = min(smin, __shfl_xor_sync(0xffffffffu, smin, o));
		smax = max(smax, __shfl_xor_sync(0xffffffffu, smax, o));
	}
	bool seen[TPL];
#pragma unroll
	for (int k = 0; k < TPL; k++) seen[k] = false;
	int maxlen = 1;
	// bounding box of the valid targets
	float3 bmin = make_float3(3.0e38f, 3.0e38f, 3.0e38f), bmax = make_float3(-3.0e38f, -3.0e38f, -3.0e38f);
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		if (tg.valid[k]) {
			bmin = make_float3(fminf(bmin.x, tg.t[k].x), fminf(bmin.y, tg.t[k].y), fminf(bmin.z, tg.t[k].z));
			bmax = make_float3(fmaxf(bmax.x, tg.t[k].x), fmaxf(bmax.y, tg.t[k].y), fmaxf(bmax.z, tg.t[k].z));
		}
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		bmin.x = fminf(bmin.x, __shfl_xor_sync(0xffffffffu, bmin.x, o));
		bmin.y = fminf(bmin.y, __shfl_xor_sync(0xffffffffu, bmin.y, o));
		bmin.z = fminf(bmin.z, __shfl_xor_sync(0xffffffffu, bmin.z, o));
		bmax.x = fmaxf(bmax.x, __shfl_xor_sync(0xffffffffu, bmax.x, o));
		bmax.y = fmaxf(bmax.y, __shfl_xor_sync(0xffffffffu, bmax.y, o));
		bmax.z = fmaxf(bmax.z, __shfl_xor_sync(0xffffffffu, bmax.z, o));
	}
	const float eps2 = fmaxf(P.soft2_f, 1e-20f);
	const float3 bc = make_float3(0.5f * (bmin.x + bmax.x), 0.5f * (bmin.y + bmax.y), 0.5f * (bmin.z + bmax.z));
	const bool single_leaves = P.leaf_size == 1;
	// far cells (fields of monopoles only): expanded about bc instead of staged
	constexpr bool USE_FAR = !POT && !DIP;
	float far2 = 3.0e38f;
	FarExp far;
	if constexpr (USE_FAR) {
		float h2 = 0.f;  // the largest squared distance of a member from bc
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			if (tg.valid[k]) {
				const float dx = tg.t[k].x - bc.x, dy = tg.t[k].y - bc.y, dz = tg.t[k].z - bc.z;
				h2 = fmaxf(h2, fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
			}
		}
#pragma unroll
		for (int o = 16; o; o >>= 1) h2 = fmaxf(h2, __shfl_xor_sync(0xffffffffu, h2, o));
		far2 = (FAR_RATIO * FAR_RATIO) * h2;
		far.zero();
	}
	const int sub = (int)lane / (32 / split);  // this lane's share of each staged list
	// Evaluation is FP32x2 in both forms.  Two targets per lane: each pair is
	// the lane's two targets against one duplicated source.  One target per
	// lane: each pair is two sources (packed by pair_pack at the flush)
	// against the duplicated target, and the two halves are added at the end.
	TgtE<2> te;
	Acc<2> E;
	if constexpr (TPL == 1) {
		te.x = make_float2(tg.t[0].x, tg.t[0].x);
		te.y = make_float2(tg.t[0].y, tg.t[0].y);
		te.z = make_float2(tg.t[0].z, tg.t[0].z);
		E.x = E.y = E.z = make_float2(0.f, 0.f);
	} else {
		to_eval(tg, te, E);
	}
	Acc<TPL>* tag = nullptr;  // selects the staging layout
	// staged sources per evaluation (a pair of sources with one target per lane)
	constexpr int PER_EV = TPL == 1 ? 2 : 1;
	// cell evaluations unrolled per lane: 8, or 4 for a split list of pairs
	// (so that the padded list fits the cell buffer)
	const int cell_unroll = (TPL == 1 && split > 1) ? 4 : 8;
	int len = 1, ncell = 0, nleaf = 0;
	uint32_t n_cells_ev = 0, n_parts_ev = 0, n_far = 0;
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
			float4 dipole = make_float4(0.f, 0.f, 0.f, 0.f);
			uint2 range = make_uint2(0u, 0u);
			int nch = 0;
			int32_t cc[8];
#pragma unroll
			for (int d = 0; d < 8; d++) cc[d] = CH_EMPTY;
			// Cells and bucket leaves load their moments from their own arrays
			// but share one opening test and one far expansion: a round whose
			// lanes hold both kinds runs that code once, not once per kind.  A
			// leaf's particle range travels in c0.x, c0.y.
			const bool is_cell = code >= 0;
			bool tested = false, opened = false;
			float r2 = 0.f;
			int4 c0 = make_int4(0, 0, 0, 0), c1 = c0;
			if (is_cell) {
				// the child codes are loaded with the cell's moments, before the
				// test, so an opened cell costs one round trip to L2, not two
				const int4* cp = reinterpret_cast<const int4*>(&T.child[8u * (uint32_t)code]);
				cell = T.f[code];
				r2 = T.r2[code];
				c0 = cp[0];
				c1 = cp[1];
				if (DIP) dipole = T.fd[code];
				tested = true;
			} else if (code != CH_EMPTY) {
				const uint32_t e = leaf_payload(code);
				if (single_leaves) {
					leafr = true;
					range = e < P.n_tree ? make_uint2(e, 1u) : T.ovf[e - P.n_tree];
				} else {
					cell = T.lf[e];
					r2 = T.lr2[e];
					const uint2 lr = T.lrange[e];  // with the moments, as for cells
					c0.x = (int)lr.x;
					c0.y = (int)lr.y;
					if (DIP) dipole = T.lfd[e];
					tested = true;
				}
			}
			if (tested) {
				if (group_accepts(bmin, bmax, bc, cell, r2, P.oap2_f)) {
					acc = cell.w != 0.f || (DIP && (dipole.x != 0.f || dipole.y != 0.f || dipole.z != 0.f));
					if (USE_FAR && acc) {
						const float fx = bc.x - cell.x, fy = bc.y - cell.y, fz = bc.z - cell.z;
						if (fmaf(fx, fx, fmaf(fy, fy, fz * fz)) > far2) {
							far.add(bc, cell);
							acc = false;
							n_far++;
						}
					}
				} else if (is_cell) {
					opened = true;
					nch = (c0.x != CH_EMPTY) + (c0.y != CH_EMPTY) + (c0.z != CH_EMPTY) + (c0.w != CH_EMPTY) +
					      (c1.x != CH_EMPTY) + (c1.y != CH_EMPTY) + (c1.z != CH_EMPTY) + (c1.w != CH_EMPTY);
				} else {
					leafr = true;
					range = make_uint2((uint32_t)c0.x, (uint32_t)c0.y);
				}
			}
			if (opened) {
				cc[0] = c0.x; cc[1] = c0.y; cc[2] = c0.z; cc[3] = c0.w;
				cc[4] = c1.x; cc[5] = c1.y; cc[6] = c1.z; cc[7] = c1.w;
			}
			leafr = leafr && range.y > 0u;  // the leaf flush relies on no staged leaf being empty
			// one warp scan for the three appends: accepted cells in bits 0-9,
			// leaf ranges in bits 10-19, children in bits 20-31 (totals <= 32,
			// <= 32 and <= 256 fit)
			int tot;
			const int packed = (acc ? 1 : 0) | ((leafr ? 1 : 0) << 10) | (nch << 20);
			const int off = warp_excl(packed, tot);
			const int co = off & 0x3FF, lo = (off >> 10) & 0x3FF, po = off >> 20;
			const int tcell = tot & 0x3FF, tleaf = (tot >> 10) & 0x3FF, tch = tot >> 20;
			if (acc) stage_src(sm.cells, ncell + co, cell, tag);
			if (DIP && acc) sm.cells[FW_CELLS + ncell + co] = dipole;
			ncell += tcell;
			if (leafr) sm.leaves[nleaf + lo] = range;
			nleaf += tleaf;
			// opened leaves that may hold members' own particles
			unsigned int hits = __ballot_sync(0xffffffffu, leafr && range.x <= smax && range.x + range.y > smin);
			while (hits) {
				const int b = __ffs(hits) - 1;
				hits &= hits - 1;
				const uint32_t rx = __shfl_sync(0xffffffffu, range.x, b);
				const uint32_t ry = __shfl_sync(0xffffffffu, range.y, b);
#pragma unroll
				for (int k = 0; k < TPL; k++) seen[k] = seen[k] || (tg.self[k] - rx < ry);
			}
			if (len + tch > FW_STACK) {
				err = POT_E_WALK;
				break;
			}
			int w = len + po;
#pragma unroll
			for (int d = 0; d < 8; d++)
				if (cc[d] != CH_EMPTY) sm.stack[w++] = cc[d];
			len += tch;
			maxlen = max(maxlen, len);
			__syncwarp();
		}
		// flush staged monopoles in whole units of the unrolled loop, so it
		// needs no remainder: a flush during the walk evaluates the whole units
		// and carries the rest (fewer than a unit) to the next; the last one
		// pads to a whole unit with zero-charge cells far outside the domain
		if (ncell >= FW_CELL_FLUSH || (done && ncell > 0)) {
			const int unit = cell_unroll * PER_EV * split;  // <= 32: the padding is one store per lane
			const int padded = done ? (ncell + unit - 1) / unit * unit : ncell / unit * unit;
			if (done && (int)lane < padded - ncell) {
				stage_src(sm.cells, ncell + lane, make_float4(64.f, 64.f, 64.f, 0.f), tag);
				if (DIP) sm.cells[FW_CELLS + ncell + lane] = make_float4(0.f, 0.f, 0.f, 0.f);
			}
			__syncwarp();
			if (TPL == 1) {
				for (int p = (int)lane; p < padded / 2; p += 32) {
					pair_pack(sm.cells, p);
					if (DIP) pair_pack_dip(sm.cells + FW_CELLS, p);
				}
				__syncwarp();
			}
			const int nev = padded / PER_EV;
			if (DIP) {  // one target per lane (creation checks the group size)
				const int stride = split, per = nev / split;
				for (int j = 0; j < per; j += 4) {
#pragma unroll
					for (int u = 0; u < 4; u++)
						eval_cell_dip<POT>(E, te, sm.cells, sm.cells + FW_CELLS, (j + u) * stride + sub);
				}
			} else if (split == 1) {
				for (int j = 0; j < nev; j += 8) {
#pragma unroll
					for (int u = 0; u < 8; u++) eval_src<false, POT>(E, te, sm.cells, j + u, eps2);
				}
			} else {
				const int per = nev / split;
				for (int j = 0; j < per; j += 4) {
#pragma unroll
					for (int u = 0; u < 4; u++) eval_src<false, POT>(E, te, sm.cells, (j + u) * split + sub, eps2);
				}
			}
			// carried cells (unpacked, fewer than 32) move to the front; the
			// ranges [padded, ncell) and [0, ncell - padded) are disjoint
			const int rem = ncell > padded ? ncell - padded : 0;
			n_cells_ev += ncell - rem;
			__syncwarp();
			if ((int)lane < rem) {
#pragma unroll
				for (int k = 0; k < TPL; k++) sm.cells[TPL * (int)lane + k] = sm.cells[TPL * (padded + (int)lane) + k];
				if (DIP) sm.cells[FW_CELLS + lane] = sm.cells[FW_CELLS + padded + lane];
			}
			ncell = rem;
			__syncwarp();
		}
		// flush staged leaves: their particles are gathered 32 at a time into
		// shared memory (dense, by a prefix sum over the leaf sizes)
		if (nleaf >= FW_LEAF_FLUSH || (done && nleaf > 0)) {
			const uint32_t c0 = (int)lane < nleaf ? sm.leaves[lane].y : 0u;
			const uint32_t c1 = (int)lane + 32 < nleaf ? sm.leaves[lane + 32].y : 0u;
			int t0, t1;
			const int e0 = warp_excl((int)c0, t0);
			const int e1 = warp_excl((int)c1, t1);
			sm.loff[lane] = (uint32_t)e0;
			sm.loff[lane + 32] = (uint32_t)(t0 + e1);
			const uint32_t total = (uint32_t)(t0 + t1);
			// start offsets of this lane's two staged leaves, ~0 for none
			const uint32_t st0 = (int)lane < nleaf ? (uint32_t)e0 : 0xFFFFFFFFu;
			const uint32_t st1 = (int)lane + 32 < nleaf ? (uint32_t)(t0 + e1) : 0xFFFFFFFFu;
			const uint32_t le_mask = (2u << lane) - 1u;  // lanes 0..lane (all for lane 31)
			int before = 0;  // staged leaves that start before this chunk
			__syncwarp();
			for (uint32_t base = 0; base < total; base += 32) {
				const uint32_t g = base + lane;
				// the staged leaves that start inside this chunk, one bit per
				// start offset (no leaf is empty, so no two share a start)
				uint32_t bits = 0u;
				if (st0 - base < 32u) bits |= 1u << (st0 - base);
				if (st1 - base < 32u) bits |= 1u << (st1 - base);
				const uint32_t starts = __reduce_or_sync(0xffffffffu, bits);
				// padding: zero charge far outside the domain
				float4 p = make_float4(64.f, 64.f, 64.f, 0.f);
				if (g < total) {
					const int a = before + __popc(starts & le_mask) - 1;  // the last leaf starting at or before g
					p = __ldg(&src32[sm.leaves[a].x + (g - sm.loff[a])]);
				}
				before += __popc(starts);
				stage_src(sm.pbuf, (int)lane, p, tag);
				__syncwarp();
				if (TPL == 1) {
					if (lane < 16) pair_pack(sm.pbuf, (int)lane);
					__syncwarp();
				}
				constexpr int nev = 32 / PER_EV;
				const uint32_t in_chunk = total - base < 32u ? total - base : 32u;
				if (split == 1 && in_chunk == 32u) {
#pragma unroll 16
					for (int m = 0; m < nev; m++) eval_src<true, POT>(E, te, sm.pbuf, m, eps2);
				} else if (split == 1) {
					// a flush's last, partial chunk: whole quads of evaluations that
					// cover its particles (the padding beyond has zero charge)
					const int need = TPL == 1 ? ((int)in_chunk + 1) / 2 : (int)in_chunk;
					const int nq = (need + 3) & ~3;  // <= nev
					for (int m = 0; m < nq; m += 4) {
#pragma unroll
						for (int u = 0; u < 4; u++) eval_src<true, POT>(E, te, sm.pbuf, m + u, eps2);
					}
				} else {
					const int per = nev / split;
#pragma unroll 8
					for (int m = 0; m < per; m++) eval_src<true, POT>(E, te, sm.pbuf, m * split + sub, eps2);
				}
				__syncwarp();
			}
			n_parts_ev += total;
			nleaf = 0;
			__syncwarp();
		}
		if (done) break;
	}
	Field<TPL> F;
	if constexpr (TPL == 1) {
		Acc<1> e1;
		e1.x = E.x.x + E.x.y;
		e1.y = E.y.x + E.y.y;
		e1.z = E.z.x + E.z.y;
		if (split > 1) {  // add the split partial fields (lanes l, l ^ 16, l ^ 8, ... share a member)
			for (int o = 16; o >= 32 / split; o >>= 1) add_xor(e1, o);
		}
		F = from_eval(e1);
	} else {
		F = from_eval(E);
	}
	if constexpr (USE_FAR) {
		far.warp_sum();
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			const float3 e = far.at(tg.t[k].x - bc.x, tg.t[k].y - bc.y, tg.t[k].z - bc.z);
			F.x[k] += e.x;
			F.y[k] += e.y;
			F.z[k] += e.z;
		}
		// the group's far cells, each expanded once
		for (int o = 16; o; o >>= 1) n_far += __shfl_xor_sync(0xffffffffu, n_far, o);
		if (n_far_cells) *n_far_cells = n_far;
	}
	// take back the members' own terms
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		if (seen[k]) {
			Acc<1> s1;
			TgtE<1> t1;
			t1.x = tg.t[k].x;
			t1.y = tg.t[k].y;
			t1.z = tg.t[k].z;
			s1.x = s1.y = s1.z = 0.f;
			const float4 own = __ldg(&src32[tg.self[k]]);
			eval_src<true, POT>(s1, t1, &own, 0, eps2);
			F.x[k] -= s1.x;
			F.y[k] -= s1.y;
			F.z[k] -= s1.z;
		}
	}
	n_eval = n_cells_ev + n_parts_ev;
	stack_max = (uint32_t)maxlen;
	return F;
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
		if (e < P.n_tree) {
			a = e;
			b = e + 1;
		} else {
			const uint2 r = T.ovf[e - P.n_tree];
			a = r.x;
			b = r.x + r.y;
		}
	} else {
		const uint2 r = T.lrange[e];
		a = r.x;
		b = r.x + r.y;
	}
}

__device__ __forceinline__ void emit_groups(unsigned int* ctr, uint2* groups, uint32_t start, uint32_t count,
                                            uint32_t gmax)
{
	while (count > 0) {
		const uint32_t c = count < gmax ? count : gmax;
		groups[atomicAdd(ctr, 1u)] = make_uint2(start, c);
		start += c;
		count -= c;
	}
}

// Target groups aligned with tree cells.  dpre[s] = due particles in slots
// [0, s).  A cell with more than gmax due particles packs its children, in
// key order, into runs of whole children holding at most gmax due particles
// (children with more start their own packing); so every group lies inside
// one parent cell and its bounding box stays compact.  (Cutting runs into
// full groups across child boundaries fills warps but widens boxes: 18 %
// more interactions and a slower walk at 1M particles.)  A group is a range
// of the due list.
// dpre == nullptr groups every particle (dpre[s] = s).
__device__ __forceinline__ uint32_t dpre_at(const uint32_t* __restrict__ dpre, uint32_t s)
{
	return dpre ? dpre[s] : s;
}

template <class G>
__device__ __forceinline__ void groups_body(G grd, const TreeDev& T, const uint32_t* __restrict__ dpre,
                                            uint2* __restrict__ groups, unsigned int* ctr, uint32_t gmax,
                                            const Params& P, RunRec* rec)
{
	if (rec->status != POT_OK) return;
	const uint32_t M = rec->n_nodes;
	for (uint32_t k = grd.id() * blockDim.x + threadIdx.x; k < M; k += grd.n() * blockDim.x) {
		const uint32_t a = T.first[k], b = T.last[k] + 1;
		const uint32_t d = dpre_at(dpre, b) - dpre_at(dpre, a);
		if (d == 0) continue;
		if (d <= gmax) {
			if (k == 0) emit_groups(ctr, groups, dpre_at(dpre, a), d, gmax);
			continue;
		}
		uint32_t run_start = 0, run = 0;
		for (int c = 0; c < 8; c++) {
			const int32_t code = T.child[8u * k + (uint32_t)c];
			if (code == CH_EMPTY) continue;
			uint32_t ca, cb;
			child_range(T, code, P, ca, cb);
			const uint32_t dc = dpre_at(dpre, cb) - dpre_at(dpre, ca);
			if (dc == 0) continue;
			if (code >= 0 && dc > gmax) {
				emit_groups(ctr, groups, run_start, run, gmax);
				run = 0;
				continue;
			}
			if (run + dc > gmax) {
				emit_groups(ctr, groups, run_start, run, gmax);
				run = 0;
			}
			if (run == 0) run_start = dpre_at(dpre, ca);
			run += dc;
		}
		emit_groups(ctr, groups, run_start, run, gmax);
	}
	// slots after the tree's (a spheroidal grain) are a group of their own
	if (grd.id() == 0 && threadIdx.x == 0 && P.n_tree < P.n) {
		const uint32_t a = dpre_at(dpre, P.n_tree), b = dpre_at(dpre, P.n);
		if (b > a) emit_groups(ctr, groups, a, b - a, gmax);
	}
}

__global__ void k_groups(TreeDev T, const uint32_t* __restrict__ dpre, uint2* __restrict__ groups, unsigned int* ctr,
                         uint32_t gmax, Params P, RunRec* rec)
{
	groups_body(GridSelf {}, T, dpre, groups, ctr, gmax, P, rec);
}

// The same groups in tree pre-order, so that the walk's warps, which take
// groups in array order, work on neighbouring groups at any one time and
// share the tree nodes they read in L2.  Three launches: each of
// GROUP_BLOCKS blocks owns a contiguous range of cells (pre-order) and counts
// the groups each cell emits (gcell, one byte a cell, and the block's total);
// one block turns the block totals into a prefix; each block then emits its
// cells' groups at the prefix plus a block scan of the cell counts, in cell
// order.  A cell's groups are the ones groups_body emits for it.
constexpr int GROUP_THREADS = 256;

template <bool EMIT>
__device__ __forceinline__ uint32_t put_groups(uint2* out, uint32_t at, uint32_t start, uint32_t count, uint32_t gmax)
{
	uint32_t k = 0;
	while (count > 0) {
		const uint32_t c = count < gmax ? count : gmax;
		if (EMIT) out[at + k] = make_uint2(start, c);
		start += c;
		count -= c;
		k++;
	}
	return k;
}

template <bool EMIT>
__device__ __forceinline__ uint32_t cell_groups(uint32_t k, const TreeDev& T, const uint32_t* __restrict__ dpre,
                                                uint32_t gmax, const Params& P, uint2* out)
{
	const uint32_t a = T.first[k], b = T.last[k] + 1;
	const uint32_t d = dpre_at(dpre, b) - dpre_at(dpre, a);
	if (d == 0) return 0;
	if (d <= gmax) return k == 0 ? put_groups<EMIT>(out, 0, dpre_at(dpre, a), d, gmax) : 0;
	uint32_t n = 0, run_start = 0, run = 0;
	for (int c = 0; c < 8; c++) {
		const int32_t code = T.child[8u * k + (uint32_t)c];
		if (code == CH_EMPTY) continue;
		uint32_t ca, cb;
		child_range(T, code, P, ca, cb);
		const uint32_t dc = dpre_at(dpre, cb) - dpre_at(dpre, ca);
		if (dc == 0) continue;
		if (code >= 0 && dc > gmax) {
			n += put_groups<EMIT>(out, n, run_start, run, gmax);
			run = 0;
			continue;
		}
		if (run + dc > gmax) {
			n += put_groups<EMIT>(out, n, run_start, run, gmax);
			run = 0;
		}
		if (run == 0) run_start = dpre_at(dpre, ca);
		run += dc;
	}
	n += put_groups<EMIT>(out, n, run_start, run, gmax);
	return n;
}

// exclusive scan over a GROUP_THREADS-thread block; *total = block sum
__device__ __forceinline__ uint32_t group_block_scan(uint32_t v, uint32_t* total)
{
	__shared__ uint32_t ws[GROUP_THREADS / 32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	uint32_t x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) ws[w] = x;
	__syncthreads();
	uint32_t before = 0, tot = 0;
#pragma unroll
	for (int k = 0; k < GROUP_THREADS / 32; k++) {
		const uint32_t t = ws[k];
		if (k < w) before += t;
		tot += t;
	}
	__syncthreads();
	*total = tot;
	return before + x - v;
}

__device__ __forceinline__ void block_cells(uint32_t M, uint32_t& k0, uint32_t& k1)
{
	k0 = (uint32_t)((uint64_t)M * blockIdx.x / gridDim.x);
	k1 = (uint32_t)((uint64_t)M * (blockIdx.x + 1) / gridDim.x);
}

__global__ void __launch_bounds__(GROUP_THREADS) k_groups_count(TreeDev T, const uint32_t* __restrict__ dpre,
                                                                uint8_t* __restrict__ gcell,
                                                                uint32_t* __restrict__ gblk, uint32_t gmax, Params P,
                                                                RunRec* rec)
{
	if (rec->status != POT_OK) return;
	uint32_t k0, k1, sum = 0;
	block_cells(rec->n_nodes, k0, k1);
	for (uint32_t k = k0 + threadIdx.x; k < k1; k += GROUP_THREADS) {
		const uint32_t n = cell_groups<false>(k, T, dpre, gmax, P, nullptr);
		gcell[k] = (uint8_t)(n < 255u ? n : 255u);  // 255: count again when emitting
		sum += n;
	}
	uint32_t tot;
	group_block_scan(sum, &tot);
	if (threadIdx.x == 0) gblk[blockIdx.x] = tot;
}

// One block: gblk[b] <- groups of the blocks before b; the slots after the
// tree's (a spheroidal grain) make the last groups; rec->n_groups the total.
__global__ void __launch_bounds__(GROUP_THREADS) k_groups_prefix(uint32_t* __restrict__ gblk, uint32_t nb,
                                                                 const uint32_t* __restrict__ dpre,
                                                                 uint2* __restrict__ groups, uint32_t gmax, Params P,
                                                                 RunRec* rec)
{
	if (rec->status != POT_OK) return;
	__shared__ uint32_t carry;
	if (threadIdx.x == 0) carry = 0;
	__syncthreads();
	for (uint32_t base = 0; base < nb; base += GROUP_THREADS) {
		const uint32_t i = base + threadIdx.x;
		const uint32_t v = i < nb ? gblk[i] : 0u;
		uint32_t tot;
		const uint32_t e = group_block_scan(v, &tot);
		const uint32_t c = carry;
		if (i < nb) gblk[i] = c + e;
		__syncthreads();
		if (threadIdx.x == 0) carry = c + tot;
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		uint32_t total = carry;
		if (P.n_tree < P.n) {
			const uint32_t a = dpre_at(dpre, P.n_tree), b = dpre_at(dpre, P.n);
			if (b > a) total += put_groups<true>(groups, total, a, b - a, gmax);
		}
		rec->n_groups = total;
	}
}

__global__ void __launch_bounds__(GROUP_THREADS) k_groups_emit(TreeDev T, const uint32_t* __restrict__ dpre,
                                                               const uint8_t* __restrict__ gcell,
                                                               const uint32_t* __restrict__ gblk,
                                                               uint2* __restrict__ groups, uint32_t gmax, Params P,
                                                               RunRec* rec)
{
	if (rec->status != POT_OK) return;
	uint32_t k0, k1;
	block_cells(rec->n_nodes, k0, k1);
	uint32_t at = gblk[blockIdx.x];
	for (uint32_t base = k0; base < k1; base += GROUP_THREADS) {
		const uint32_t k = base + threadIdx.x;
		uint32_t n = k < k1 ? gcell[k] : 0u;
		if (n == 255u) n = cell_groups<false>(k, T, dpre, gmax, P, nullptr);
		uint32_t tot;
		const uint32_t off = group_block_scan(n, &tot);
		if (n) cell_groups<true>(k, T, dpre, gmax, P, groups + at + off);
		at += tot;
	}
}

// The point where a target's field is evaluated: for the Boris step the
// position drifted half a step, x + (dt tss / 2) v (pot.c:2478-2485); for
// the stages of the other integrators the position itself.
template <int STG>
__device__ __forceinline__ double3 eval_point(const double4 p, const double4* __restrict__ vel, uint32_t s,
                                              const Params& P)
{
	if (STG == 0) {
		const double4 v = vel[s];
		const double half = 0.5 * (P.dt * (double)P.tss[(int)p.w]);
		return make_double3(fma(half, v.x, p.x), fma(half, v.y, p.y), fma(half, v.z, p.z));
	}
	return make_double3(p.x, p.y, p.z);
}

// Per-launch state of one run's push: the grain (its position for the
// absorption test, its charge) and the scale of the walk's FP32 sums.
struct PushCtx {
	const float4* srcf;
	double gx, gy, gz, qg, escale;
	bool grain_due, absorb_on;
};

template <int STG>
__device__ __forceinline__ PushCtx push_ctx(const double4* __restrict__ pos, const float4* __restrict__ src32,
                                            const Params& P, const RunRec* rec, const StageBufs& sb)
{
	PushCtx c;
	const unsigned long long t_step = rec->t_steps;
	c.grain_due = rec->grain_due != 0;
	c.absorb_on = !(P.flags & FLAG_NO_GRAIN) && t_step >= P.t_settle;
	c.gx = rec->grain_pos[0];
	c.gy = rec->grain_pos[1];
	c.gz = rec->grain_pos[2];
	if (STG == 2 && c.grain_due && rec->grain_slot < P.n) {
		const double4 gp = pos[rec->grain_slot];  // the grain's intermediate position
		c.gx = gp.x; c.gy = gp.y; c.gz = gp.z;
	}
	c.srcf = STG == 2 ? sb.src32b : src32;
	c.qg = (double)rec->grain_q;
	c.escale = QE / (P.k4 * P.rad * P.rad);
	return c;
}

// One target group grp = (first entry of the due list, count): the warp's
// walk for the whole group, then each member's push, absorption and boundary
// test.  Adds to the lane's interaction and push counts and the deepest
// stack; returns the walk's status (a member that fails leaves the group's
// pushes undone).
template <int TPL, int STG, bool DIP>
__device__ __forceinline__ int push_group(uint2 grp, double4* __restrict__ pos, double4* __restrict__ vel,
                                          const TreeDev& T, const float4* __restrict__ src32,
                                          const uint32_t* __restrict__ due_list, uint32_t* __restrict__ rein_list,
                                          const Params& P, RunRec* rec, const double4* __restrict__ src64,
                                          const StageBufs& sb, const PushCtx& pc, FastSmem<TPL, DIP>& sm,
                                          unsigned long long& n_inter, unsigned long long& n_push,
                                          uint32_t& stack_max, unsigned long long& n_far)
{
	Targets<TPL> tg;
	uint32_t slot[TPL];
	// small groups split the warp (see group_walk): lanes past the
	// first 32 / split hold copies of members and push nothing
	const int split = TPL == 1 ? (grp.y <= 8 ? 4 : (grp.y <= 16 ? 2 : 1)) : 1;
	const uint32_t width = 32u / (uint32_t)split;
	const bool owner = lane_f() < width;
	// the FP64 evaluation point (half-drifted for the Boris step) is
	// recomputed after the walk from the same state with the same
	// operations, so it is not held in registers through the walk
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		const uint32_t m = (lane_f() & (width - 1u)) + 32u * k;
		tg.valid[k] = m < grp.y;
		slot[k] = 0xFFFFFFFFu;
		double3 h = make_double3(P.rad, P.rad, P.rad);
		if (tg.valid[k]) {
			slot[k] = due_list[grp.x + m];
			h = eval_point<STG>(pos[slot[k]], vel, slot[k], P);
		}
		tg.self[k] = slot[k];
		tg.t[k] = make_float3((float)((h.x - P.rad) * P.inv_rad), (float)((h.y - P.rad) * P.inv_rad),
		                      (float)((h.z - P.rad) * P.inv_rad));
	}
	uint32_t ne = 0, depth = 0, nf = 0;
	int err = POT_OK;
	const Field<TPL> ef = group_walk<TPL, false, DIP>(tg, T, pc.srcf, P, sm, ne, depth, err, split, &nf);
	stack_max = max(stack_max, depth);
	if (err != POT_OK) return err;
	if (lane_f() == 0) n_far += nf;
#pragma unroll
	for (int k = 0; k < TPL; k++) {
		if (!tg.valid[k] || !owner) continue;
		const uint32_t s = slot[k];
		const double4 p = pos[s];
		double4 v = vel[s];
		const int sp = (int)p.w;
		const double dt = P.dt * (double)P.tss[sp];
		// the evaluation point as eval_point computes it, from the same values
		const double3 hk = STG == 0 ? make_double3(fma(0.5 * dt, v.x, p.x), fma(0.5 * dt, v.y, p.y),
		                                           fma(0.5 * dt, v.z, p.z))
		                            : make_double3(p.x, p.y, p.z);
		n_inter += ne;
		if (STG != 1) n_push++;
		double E[3] = { (double)ef.x[k] * pc.escale, (double)ef.y[k] * pc.escale, (double)ef.z[k] * pc.escale };
		if (P.shape && sp != SP_DUST) {
			// the spheroid's own field in FP64 (pot-spheroid.c:1815-1819)
			double Eg[3];
			spheroid_field(P, pc.qg, dsub(hk.x, pc.gx), dsub(hk.y, pc.gy), dsub(hk.z, pc.gz), Eg);
			E[0] += Eg[0];
			E[1] += Eg[1];
			E[2] += Eg[2];
		}
		const double charge = sp == SP_DUST ? pc.qg : (sp == SP_ION ? 1.0 : -1.0);
		const double qom = (QE * charge) / mass_of(sp, P);
		if (STG == 1) {
			const double3 a1 = accel_lorentz(E, v, qom, P);
			double4 pm = p;
			half_first(pm, v, a1, dt, P);
			pos[s] = pm;
			vel[s] = v;
			sb.acc[s] = make_double4(a1.x, a1.y, a1.z, 0.0);
			sb.src32b[s] = make_float4((float)((pm.x - P.rad) * P.inv_rad), (float)((pm.y - P.rad) * P.inv_rad),
			                           (float)((pm.z - P.rad) * P.inv_rad), src32[s].w);
			sb.src64b[s] = make_double4(pm.x, pm.y, pm.z, src64[s].w);
			continue;
		}
		double3 xn;
		if (STG == 0) {
			boris(v, hk, E, qom, dt, P, xn);
		} else {
			const double4 a = sb.acc[s];
			half_second(xn, v, p, make_double3(a.x, a.y, a.z), accel_lorentz(E, v, qom, P), dt, P);
		}
		uint32_t reason = 0;
		if (!pc.grain_due)
			reason = after_push(sp, STG == 0 ? p : src64[s], xn, v, P, rec, pc.absorb_on, pc.gx, pc.gy, pc.gz);
		pos[s] = make_double4(xn.x, xn.y, xn.z, p.w);
		vel[s] = v;
		if (reason) rein_list[atomicAdd(&rec->n_rein, 1u)] = s | (reason << 30);
	}
	return POT_OK;
}

// The lanes' interaction and push counts, far cells and deepest stack into
// the run record.
__device__ __forceinline__ void push_stats(RunRec* rec, unsigned long long n_inter, unsigned long long n_push,
                                           uint32_t stack_max, unsigned long long n_far)
{
	unsigned long long a = n_inter, b = n_push, f = n_far;
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		a += __shfl_xor_sync(0xffffffffu, a, o);
		b += __shfl_xor_sync(0xffffffffu, b, o);
		f += __shfl_xor_sync(0xffffffffu, f, o);
	}
	if (lane_f() == 0) {
		if (a) atomicAdd(&rec->interactions, a);
		if (b) atomicAdd(&rec->n_pushed, b);
		if (f) atomicAdd(&rec->far_cells, f);
		if (stack_max) atomicMax(&rec->stack_max, stack_max);
	}
}

// STG as in k_push_plain: 0 the Boris step; 1 and 2 the two halves of the
// non-Boris integrators (stage 2 walks over the intermediate sources).
// Persistent: each warp takes the next group from the run's work counter.
template <int TPL, int STG, bool DIP = false>
__global__ void __launch_bounds__(FW_WARPS * 32, fw_push_blocks(TPL))
k_push_fast(double4* __restrict__ pos, double4* __restrict__ vel, TreeDev T, const float4* __restrict__ src32,
            const uint32_t* __restrict__ due_list, const uint2* __restrict__ groups, uint32_t* __restrict__ rein_list,
            Params P, RunRec* rec, const double4* __restrict__ src64, StageBufs sb)
{
	__shared__ FastSmem<TPL, DIP> smem[FW_WARPS];
	FastSmem<TPL, DIP>& sm = smem[threadIdx.x >> 5];
	// warp-uniform: another warp may set the status meanwhile
	if (__shfl_sync(0xffffffffu, lane_f() == 0 ? rec->status : 0, 0) != POT_OK) return;
	const uint32_t n_groups = rec->n_groups;
	const PushCtx pc = push_ctx<STG>(pos, src32, P, rec, sb);
	unsigned long long n_inter = 0, n_push = 0, n_far = 0;
	uint32_t stack_max = 0;
	for (;;) {
		uint32_t g = 0;
		if (lane_f() == 0) g = atomicAdd(&rec->work_ctr, 1u);
		g = __shfl_sync(0xffffffffu, g, 0);
		if (g >= n_groups) break;
		const int err = push_group<TPL, STG, DIP>(groups[g], pos, vel, T, src32, due_list, rein_list, P, rec, src64,
		                                          sb, pc, sm, n_inter, n_push, stack_max, n_far);
		if (err != POT_OK) {
			if (lane_f() == 0) set_status(rec, err);
			break;
		}
	}
	push_stats(rec, n_inter, n_push, stack_max, n_far);
}

template <int TPL, bool DIP = false>
__global__ void __launch_bounds__(FW_WARPS * 32) k_field_query_fast(TreeDev T, const float4* __restrict__ src32,
                                                                   const double* __restrict__ xyz,
                                                                   const uint32_t* __restrict__ self_slot,
                                                                   uint32_t nq, double* __restrict__ E, Params P,
                                                                   RunRec* rec)
{
	__shared__ FastSmem<TPL, DIP> smem[FW_WARPS];
	FastSmem<TPL, DIP>& sm = smem[threadIdx.x >> 5];
	const uint32_t gsize = 32u * TPL;
	const uint32_t n_groups = (nq + gsize - 1) / gsize;
	const double escale = QE / (P.k4 * P.rad * P.rad);
	for (uint32_t g = blockIdx.x * FW_WARPS + (threadIdx.x >> 5); g < n_groups; g += gridDim.x * FW_WARPS) {
		Targets<TPL> tg;
		uint32_t q[TPL];
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			q[k] = g * gsize + lane_f() + 32u * k;
			tg.valid[k] = q[k] < nq;
			tg.t[k] = make_float3(0.f, 0.f, 0.f);
			tg.self[k] = 0xFFFFFFFFu;
			if (tg.valid[k]) {
				const uint32_t j = q[k];
				tg.t[k] = make_float3((float)((xyz[3 * j] - P.rad) * P.inv_rad),
				                      (float)((xyz[3 * j + 1] - P.rad) * P.inv_rad),
				                      (float)((xyz[3 * j + 2] - P.rad) * P.inv_rad));
				tg.self[k] = self_slot[j];
			}
		}
		uint32_t ne = 0, depth = 0;
		int err = POT_OK;
		const Field<TPL> ef = group_walk<TPL, false, DIP>(tg, T, src32, P, sm, ne, depth, err);
		if (err != POT_OK && lane_f() == 0) set_status(rec, err);
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			if (!tg.valid[k]) continue;
			const uint32_t j = q[k];
			double Eg[3] = { 0.0, 0.0, 0.0 };
			if (P.shape && self_slot[j] != rec->grain_slot) {
				spheroid_field(P, (double)rec->grain_q, dsub(xyz[3 * j], rec->grain_pos[0]),
				               dsub(xyz[3 * j + 1], rec->grain_pos[1]), dsub(xyz[3 * j + 2], rec->grain_pos[2]), Eg);
			}
			E[3 * j] = (double)ef.x[k] * escale + Eg[0];
			E[3 * j + 1] = (double)ef.y[k] * escale + Eg[1];
			E[3 * j + 2] = (double)ef.z[k] * escale + Eg[2];
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

uint32_t group_blocks() { return (uint32_t)sm_count_fast() * 4u; }

void launch_groups(const TreeDev& T, const uint32_t* dpre, uint2* groups, uint8_t* gcell, uint32_t* gblk,
                   const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	cudaMemsetAsync(&rec->n_groups, 0, sizeof(unsigned int), s);
	if (!gcell) {  // one launch, groups in the order their cells finish
		ScopedKernel k(tm, "groups");
		k_groups<<<sm_count_fast() * 4, 256, 0, s>>>(T, dpre, groups, &rec->n_groups, P.group_max, P, rec);
		return;
	}
	const uint32_t nb = group_blocks();
	ScopedKernel k(tm, "groups", 3);
	k_groups_count<<<nb, GROUP_THREADS, 0, s>>>(T, dpre, gcell, gblk, P.group_max, P, rec);
	k_groups_prefix<<<1, GROUP_THREADS, 0, s>>>(gblk, nb, dpre, groups, P.group_max, P, rec);
	k_groups_emit<<<nb, GROUP_THREADS, 0, s>>>(T, dpre, gcell, gblk, groups, P.group_max, P, rec);
}

// compute_epe (pot.c:2771-2804), fast form: groups of up to 32 TPL over
// every particle, the group walk accumulating potentials; per-group partial
// sums of q e phi per species, summed in group order by k_epe_final.
template <int TPL, bool DIP = false>
__global__ void __launch_bounds__(FW_WARPS * 32) k_epe_fast(const double4* __restrict__ pos, TreeDev T,
                                                           const float4* __restrict__ src32,
                                                           const double4* __restrict__ src64,
                                                           const uint2* __restrict__ groups,
                                                           double* __restrict__ partial, Params P, RunRec* rec)
{
	__shared__ FastSmem<TPL, DIP> smem[FW_WARPS];
	FastSmem<TPL, DIP>& sm = smem[threadIdx.x >> 5];
	// warp-uniform: another warp may set the status meanwhile
	if (__shfl_sync(0xffffffffu, lane_f() == 0 ? rec->status : 0, 0) != POT_OK) return;
	const uint32_t n_groups = rec->n_groups_all;
	const uint32_t gs = rec->grain_slot;
	const double pscale = QE / (P.k4 * P.rad);
	for (;;) {
		uint32_t g = 0;
		if (lane_f() == 0) g = atomicAdd(&rec->work_ctr2, 1u);
		g = __shfl_sync(0xffffffffu, g, 0);
		if (g >= n_groups) break;
		const uint2 grp = groups[g];
		Targets<TPL> tg;
		float qme[TPL];
		const int split = TPL == 1 ? (grp.y <= 8 ? 4 : (grp.y <= 16 ? 2 : 1)) : 1;
		const uint32_t width = 32u / (uint32_t)split;
		const bool owner = lane_f() < width;
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			const uint32_t m = (lane_f() & (width - 1u)) + 32u * k;
			tg.valid[k] = m < grp.y;
			tg.self[k] = tg.valid[k] ? grp.x + m : 0xFFFFFFFFu;
			const float4 me = tg.valid[k] ? src32[grp.x + m] : make_float4(0.f, 0.f, 0.f, 0.f);
			tg.t[k] = make_float3(me.x, me.y, me.z);
			qme[k] = me.w;
		}
		uint32_t ne = 0, depth = 0;
		int err = POT_OK;
		const Field<TPL> f = group_walk<TPL, true, DIP>(tg, T, src32, P, sm, ne, depth, err, split);
		if (err != POT_OK) {
			if (lane_f() == 0) set_status(rec, err);
			break;
		}
		double acc[3] = { 0.0, 0.0, 0.0 };
#pragma unroll
		for (int k = 0; k < TPL; k++) {
			if (!tg.valid[k] || !owner) continue;
			const uint32_t slot = tg.self[k];
			double phi = (double)f.x[k] * pscale;
			if (slot == gs) {
				rec->phi_grain = phi;
			} else {
				if (P.shape) {  // the spheroid's own potential, FP64 (pot-spheroid.c:2107-2109)
					const double4 p = src64[slot];
					phi += spheroid_phi(P, (double)rec->grain_q, dsub(p.x, rec->grain_pos[0]),
					                    dsub(p.y, rec->grain_pos[1]), dsub(p.z, rec->grain_pos[2]));
				}
				acc[(int)pos[slot].w] += (QE * (double)qme[k]) * phi;
			}
		}
#pragma unroll
		for (int k = 0; k < 3; k++)
			for (int o = 16; o; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
		if (lane_f() == 0)
			for (int k = 0; k < 3; k++) partial[3 * g + k] = acc[k];
	}
}

void launch_epe_fast(const double4* pos, const TreeDev& T, const float4* src32, const double4* src64,
                     uint2* groups_all, double* partial, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	cudaMemsetAsync(&rec->n_groups_all, 0, sizeof(unsigned int), s);
	cudaMemsetAsync(&rec->work_ctr2, 0, sizeof(unsigned int), s);
	ScopedKernel k(tm, "epe_fast", 2);
	const bool two = P.group_max > 32;
	k_groups<<<sm_count_fast() * 4, 256, 0, s>>>(T, nullptr, groups_all, &rec->n_groups_all, two ? 64u : 32u, P,
	                                              rec);
	if (two) {
		k_epe_fast<2><<<sm_count_fast() * 6, FW_WARPS * 32, 0, s>>>(pos, T, src32, src64, groups_all, partial, P,
		                                                            rec);
	} else if (T.fd) {
		k_epe_fast<1, true><<<sm_count_fast() * 6, FW_WARPS * 32, 0, s>>>(pos, T, src32, src64, groups_all, partial,
		                                                                  P, rec);
	} else {
		k_epe_fast<1><<<sm_count_fast() * 6, FW_WARPS * 32, 0, s>>>(pos, T, src32, src64, groups_all, partial, P,
		                                                            rec);
	}
}

template <int STG>
static void push_fast_stage(double4* pos, double4* vel, const TreeDev& T, const float4* src32, const double4* src64,
                            const uint32_t* due_list, const uint2* groups, uint32_t* rein_list, const Params& P,
                            RunRec* rec, const StageBufs& sb, cudaStream_t s)
{
	const int nb = sm_count_fast() * 6;
	if (P.group_max > 32) {
		k_push_fast<2, STG><<<nb, FW_WARPS * 32, 0, s>>>(pos, vel, T, src32, due_list, groups, rein_list, P, rec,
		                                                 src64, sb);
	} else if (T.fd) {  // DIPOLES
		k_push_fast<1, STG, true><<<nb, FW_WARPS * 32, 0, s>>>(pos, vel, T, src32, due_list, groups, rein_list, P,
		                                                       rec, src64, sb);
	} else {
		k_push_fast<1, STG><<<nb, FW_WARPS * 32, 0, s>>>(pos, vel, T, src32, due_list, groups, rein_list, P, rec,
		                                                 src64, sb);
	}
}

void launch_push_fast(double4* pos, double4* vel, const TreeDev& T, const float4* src32, const double4* src64,
                      const uint32_t* due_list, const uint2* groups, uint32_t* rein_list, const Params& P,
                      RunRec* rec, const StageBufs& sb, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, sb.stage == 0 ? "walk_push_fast" : (sb.stage == 1 ? "walk_half1_fast" : "walk_half2_fast"));
	if (sb.stage == 0) {
		push_fast_stage<0>(pos, vel, T, src32, src64, due_list, groups, rein_list, P, rec, sb, s);
	} else if (sb.stage == 1) {
		push_fast_stage<1>(pos, vel, T, src32, src64, due_list, groups, rein_list, P, rec, sb, s);
	} else {
		push_fast_stage<2>(pos, vel, T, src32, src64, due_list, groups, rein_list, P, rec, sb, s);
	}
}

void launch_field_query_fast(const TreeDev& T, const float4* src32, const double* xyz, const uint32_t* self_slot,
                             uint32_t nq, double* E, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "field_query_fast");
	const uint32_t gsize = P.group_max > 32 ? 64u : 32u;
	const uint32_t groups = (nq + gsize - 1) / gsize;
	uint32_t nb = (groups + FW_WARPS - 1) / FW_WARPS;
	if (nb == 0) nb = 1;
	if (gsize == 64) {
		k_field_query_fast<2><<<nb, FW_WARPS * 32, 0, s>>>(T, src32, xyz, self_slot, nq, E, P, rec);
	} else {
		if (T.fd)
			k_field_query_fast<1, true><<<nb, FW_WARPS * 32, 0, s>>>(T, src32, xyz, self_slot, nq, E, P, rec);
		else
			k_field_query_fast<1><<<nb, FW_WARPS * 32, 0, s>>>(T, src32, xyz, self_slot, nq, E, P, rec);
	}
}

}  // namespace pot

// ---------------------------------------------------------------------------
// packed batch: target groups and the walk of every member in one launch
// ---------------------------------------------------------------------------
namespace pot {

__global__ void kp_groups(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_GROUPS], B.M);
	const MemberView& v = B.mv[sb.m];
	groups_body(GridSeg { sb.id, sb.n }, v.T, v.due_prefix, v.groups, &v.rec->n_groups, v.P.group_max, v.P, v.rec);
}

// gpre[m] = target groups of members 0..m-1 (a member whose status is set
// contributes none); the walk's work counter is reset.  One block.
__global__ void __launch_bounds__(1024) kp_group_prefix(PackDev B)
{
	__shared__ uint32_t carry;
	if (threadIdx.x == 0) {
		carry = 0;
		*B.ctr = 0u;
	}
	__syncthreads();
	for (uint32_t base = 0; base < B.M; base += blockDim.x) {
		const uint32_t m = base + threadIdx.x;
		uint32_t c = 0;
		if (m < B.M) {
			const RunRec* r = B.mv[m].rec;
			c = r->status == POT_OK ? r->n_groups : 0u;
		}
		// block-wide inclusive scan of c, warp by warp
		__shared__ uint32_t wsum[32];
		uint32_t x = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
			if ((threadIdx.x & 31) >= (unsigned)o) x += t;
		}
		if ((threadIdx.x & 31) == 31) wsum[threadIdx.x >> 5] = x;
		__syncthreads();
		if (threadIdx.x < 32) {
			uint32_t y = threadIdx.x < (blockDim.x >> 5) ? wsum[threadIdx.x] : 0u;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const uint32_t t = __shfl_up_sync(0xffffffffu, y, o);
				if (threadIdx.x >= (unsigned)o) y += t;
			}
			wsum[threadIdx.x] = y;
		}
		__syncthreads();
		const uint32_t incl = x + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0u) + carry;
		if (m < B.M) B.gpre[m] = incl - c;
		__syncthreads();
		if (threadIdx.x == blockDim.x - 1) carry = incl;
		__syncthreads();
	}
	if (threadIdx.x == 0) B.gpre[B.M] = carry;
}

// The walk and push of every member's groups: each warp takes the next
// group of the whole batch, finds its member in gpre and runs it with that
// member's tree, state and record; counts go to the member's record.
template <int TPL>
__global__ void __launch_bounds__(FW_WARPS * 32, fw_push_blocks(TPL)) kp_push_fast(PackDev B, int k)
{
	__shared__ FastSmem<TPL, false> smem[FW_WARPS];
	FastSmem<TPL, false>& sm = smem[threadIdx.x >> 5];
	const uint32_t total = B.gpre[B.M];
	const StageBufs sb { 0, nullptr, nullptr, nullptr };
	for (;;) {
		uint32_t g = 0;
		if (lane_f() == 0) g = atomicAdd(B.ctr, 1u);
		g = __shfl_sync(0xffffffffu, g, 0);
		if (g >= total) break;
		uint32_t lo = 0, hi = B.M;  // gpre[lo] <= g < gpre[hi]
		while (hi - lo > 1) {
			const uint32_t mid = (lo + hi) >> 1;
			if (B.gpre[mid] <= g) lo = mid; else hi = mid;
		}
		const MemberView& v = B.mv[lo];
		RunRec* rec = v.rec;
		// warp-uniform: another warp may set the status meanwhile
		if (__shfl_sync(0xffffffffu, lane_f() == 0 ? rec->status : 0, 0) != POT_OK) continue;
		const uint32_t b = pack_out(v, k);
		const PushCtx pc = push_ctx<0>(v.pos[b], v.src32, v.P, rec, sb);
		unsigned long long n_inter = 0, n_push = 0, n_far = 0;
		uint32_t stack_max = 0;
		const int err = push_group<TPL, 0, false>(v.groups[g - B.gpre[lo]], v.pos[b], v.vel[b], v.T, v.src32,
		                                          v.due_list, v.rein_list, v.P, rec, v.src64, sb, pc, sm, n_inter,
		                                          n_push, stack_max, n_far);
		if (err != POT_OK && lane_f() == 0) set_status(rec, err);
		push_stats(rec, n_inter, n_push, stack_max, n_far);
	}
}

void pack_groups(const PackDev& B, cudaStream_t s)
{
	kp_groups<<<B.blocks[PS_GROUPS], 256, 0, s>>>(B);
	kp_group_prefix<<<1, 1024, 0, s>>>(B);
}

void pack_push(const PackDev& B, int k, uint32_t tpl, cudaStream_t s)
{
	const int nb = sm_count_fast() * 5;
	if (tpl == 2) kp_push_fast<2><<<nb, FW_WARPS * 32, 0, s>>>(B, k);
	else kp_push_fast<1><<<nb, FW_WARPS * 32, 0, s>>>(B, k);
}

}  // namespace pot
