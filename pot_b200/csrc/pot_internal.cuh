// Shared device definitions for the sm_100a particle-loop kernels.
//
// Layout in HBM (one run):
//   particle state, Morton order, double-buffered across the per-step
//   reorder:  pos[s] = (x, y, z, species) double4, vel[s] = (vx, vy, vz, 0)
//   double4, pid[s] = index in the reference's particle array (uint32);
//   tree sources, written by the reorder: src64[s] = (x, y, z, charge) and,
//   for the fast form, src32[s] = (x - c, y - c, z - c, charge) float4 with c
//   the domain centre;
//   internal tree nodes in pre-order (parents before children, children in
//   key order), structure of arrays.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pot_gpu.h"

namespace pot {

// Physical constants of pot.c:278-282 (SI).  PI/SQRT_PI are the 15-digit
// doubles prng.h:10-15 defines, which are the ones in force in pot.c.
constexpr double KB = 1.38065e-23;
constexpr double EPSILON0 = 8.85419e-12;
constexpr double QE = 1.6021766e-19;
constexpr double ME = 9.109383e-31;
constexpr double MIME = 1836.15;
constexpr double PI_REF = 3.14159265358979;
constexpr double SQRT_PI_REF = 1.77245385090552;
// MASS[] of pot.c:292: each a double constant widened to long double.
constexpr double MASS_DUST = 1.67e-12;
constexpr double MASS_ION = MIME * ME;
constexpr double MASS_E = ME;

enum Species : int { SP_DUST = 0, SP_ION = 1, SP_E = 2 };

// Tree child codes: >= 0 internal node; CH_EMPTY; otherwise a leaf whose
// payload index is -2 - code (a particle slot for leaf size 1, an entry of
// the leaf table 8 * parent + digit for bucket leaves).
constexpr int32_t CH_EMPTY = -1;
__host__ __device__ inline int32_t leaf_code(uint32_t i) { return -2 - (int32_t)i; }
__host__ __device__ inline uint32_t leaf_payload(int32_t c) { return (uint32_t)(-2 - c); }

// The reference's child member order (pot.c:323-330) as octal digits
// (gx << 2 | gy << 1 | gz): gxlylz, gxlygz, lxlylz, lxlygz, lxgylz, lxgygz,
// gxgylz, gxgygz.  Moments and walks visit children in this order.
__host__ __device__ inline int slot_digit(int s)
{
	return (0x76321054 >> (4 * s)) & 0xF;
}

constexpr int MAX_LEVELS = 21;     // 63-bit keys, 3 bits per level
constexpr int WALK_STACK = 400;    // MAX_PATH_LEN, pot.c:196
// Leaf size 1 cannot hold two particles that share all 21 key levels (closer
// than 2R / 2^21 in every axis); such a level-21 cell becomes a bucket in a
// small overflow table, leaf payload n + j, and sets warn bit 0.
constexpr uint32_t OVF_CAP = 4096;
// Fast form: largest target group per warp (two targets per lane).
constexpr uint32_t GROUP_MAX = 64;
constexpr uint32_t FLAG_SCEPTIC = POT_CFG_SCEPTIC;
constexpr uint32_t FLAG_NO_GRAIN = POT_CFG_DISABLE_GRAIN;
constexpr uint32_t FLAG_DIPOLES = POT_CFG_DIPOLES;
constexpr uint32_t FLAG_POIS = POT_CFG_POIS_IONS;
constexpr uint32_t WARN_WALL = 128u;     // OUT_BOUNCE: a particle in the wall moving inwards
constexpr uint32_t WARN_POISSON = 256u;  // the Poisson variate's iteration cap
constexpr uint32_t WARN_CHI_CAP = 512u;  // POT_OPT_CHI_CAP: the sampler's edge potential was capped
constexpr uint32_t FLAG_CHI_CAP = 0x100u;  // Params.flags: POT_OPT_CHI_CAP (above the run's POT_CFG_* bits)

// Device-resident record of one run; the host reads it only at sync points.
struct RunRec {
	unsigned long long t_steps;
	long long grain_q;
	double grain_m;
	double grain_pos[3];
	double grain_vel[3];
	unsigned long long tot_absor_e;
	double chi_b;
	int status;              // first error (sticky), POT_OK otherwise
	unsigned int grain_slot; // grain's slot in Morton order this step
	// per step, reset by the keys kernel
	unsigned int n_due;
	unsigned int n_rein;
	unsigned int n_nodes;
	unsigned int work_ctr;   // dynamic work distribution counter
	unsigned int work_ctr2;  // second counter (potential-energy walk)
	unsigned int stack_max;  // deepest fast-walk stack this step
	unsigned int grain_due;
	unsigned int warn;       // non-fatal conditions (bit 0: key collision at 21 levels)
	unsigned int n_overflow; // deepest-level buckets of a leaf-size-1 tree this build
	unsigned int n_groups;   // fast form: target groups this step
	unsigned int n_groups_all;  // fast form: groups over every particle (potential energies)
	long long dq;
	unsigned long long de;
	unsigned long long nabs_ion;
	unsigned long long nabs_e;
	long long sumv_ion[3];   // fixed point, 2^-20 m/s
	long long sumv_e[3];
	unsigned long long interactions;
	unsigned long long n_pushed;
	unsigned long long far_cells;  // fast form: far cells expanded about their group's centre
	double epe[3];           // potential energies of the last step that computed them (J)
	double phi_grain;        // potential at the grain from every other particle (V)
	unsigned int epe_step;   // 1 when this step computes them
	unsigned int epe_pad;
	long long q_sum;         // sum over completed steps of the grain charge after each step (moving means)
	unsigned int n_collected;  // Poisson ion collection: charges added this step
	unsigned int n_wall;       // OUT_BOUNCE: particles outside moving inwards this step
	unsigned int n_bounced;    // OUT_BOUNCE: particles bounced this step
	unsigned int pad_v;
	double ion_temp;           // cached ion temperature of the Poisson collection (Proc.Ti)
};

constexpr double VFIX = 1048576.0;  // 2^20

// Per-step statistics ring entry (read back by the host).
struct StepHist {
	unsigned long long t_steps;
	long long grain_q;
	long long dq;
	unsigned long long de;
	unsigned long long n_absorbed;
	unsigned long long n_reinjected;
	unsigned long long n_pushed;
	unsigned long long interactions;
	unsigned long long n_nodes;
	unsigned long long far_cells;
	double chi_b;
	int status;
	int pad;
	double epe[3];
};
constexpr int HIST = 64;
constexpr int EPE_BLOCKS = 592;  // per-block partial sums of the potential-energy walks (4 x 148)

// Constant per-run parameters, passed by value to every kernel.
struct Params {
	uint32_t n;           // particles in the state arrays (= tree sources)
	uint32_t n_total;     // Run.N
	uint32_t n_ions;      // ions carry original indices 1..n_ions
	uint32_t r_pix;       // Run.r
	uint32_t leaf_size;
	uint32_t flags;
	uint32_t tss[3];
	uint32_t form;
	uint32_t max_level;  // deepest level (leaf cells): 21 in the plain form, 16 in the fast form
	uint32_t key_bits;   // low key bits left unsorted: 0 plain, 15 fast (levels 17-21)
	uint32_t group_max;  // fast form: targets per warp group, 32 or 64
	uint64_t seed;
	unsigned long long t_settle;  // first step with t*dt > settle (long double test on the host)
	double dt, mpp, rad, root_w;  // rad = r*mpp, root_w = 2.0*r*mpp (pot.c:1476)
	double inv_rad;
	double soft, soft2;
	double a;
	double Te, Ti, x_drift;
	double oap2;          // OAP*OAP
	double k4;            // 4*PI*EPSILON0 as pot.c folds it
	double Bmag;
	double bhat[3];
	double sigma_i, sigma_e;  // Maxwellian sd per species, pot.c:675-681
	double vn_i, vn_e;        // SCEPTIC normalisation speeds, pot.c:517-524
	double Rol;               // R / Debye length of pot.c:577-579
	float oap2_f;
	float soft2_f;        // (soft / rad)^2: FP32 walk works in units of the domain radius
	uint32_t n_tree;      // tree sources: slots [0, n_tree); n - 1 with a spheroidal grain (kept last, outside)
	uint32_t shape;       // grain: 0 sphere (pot.c), 1 prolate, 2 oblate spheroid (pot-spheroid.c)
	double m_ion;         // MASS[ION] = MIME * ME; MIME 1836.15, or 1836.153 in pot-spheroid.c:61
	double max_lin_dev;   // integrate_for_alpha tolerance: 0.01, or 0.1 in pot-spheroid.c:457
	// spheroid constants (host libm, in the reference's operation order):
	// phi_const = ((QE q) s_num) / s_den_*, s_fc_* the focal distances of the
	// field (pot-spheroid.c:1702-1715) and potential (1926-1946, 2056-2069) forms
	double s_A, s_fc_f, s_fc_p, s_num, s_den_f, s_den_p;
	double s_thr;         // a^2 A^(4/3): surface x^2 + A^2 rho^2 = a^2 A^(4/3)
	uint32_t s_tilted;    // symmetry axis other than x (an extension of the reference)
	uint32_t chi_ranks;   // azimuths averaged for chi_b (ranks of an MPI run), >= 1
	double s_ax[3], s_e1[3], s_e2[3];  // spheroid frame
	double B[3];          // EXTERNAL_B_X/Y/Z as given (non-Boris accelerations)
	double bounce;        // OUT_BOUNCE coefficient of restitution; 0 = reinjection at the wall
	double pos_rate_const;  // Poisson ion collection: constant part of the rate (pot.c:4253-4255)
	uint32_t integrator;  // POT_INT_*
	uint32_t pad_v;
};

// ---- exactly rounded double helpers (no FMA contraction) ---------------
// The reference is compiled for x86-64 SSE2, where a*b+c is two rounded
// operations.  Parity-critical arithmetic (tree moments, the opening test,
// the absorption test) uses these so nvcc cannot fuse them.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsq3(double x, double y, double z)
{
	return dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z));
}

// ---- Philox4x32-10 (Salmon et al., SC'11) -------------------------------
__host__ __device__ inline void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
	for (int r = 0; r < 10; r++) {
		const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
		const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
		const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
		const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
		c[0] = n0;
		c[1] = (uint32_t)p1;
		c[2] = n2;
		c[3] = (uint32_t)p0;
		k0 += 0x9E3779B9u;
		k1 += 0xBB67AE85u;
	}
}

// Sequential uint32 stream for one (particle id, step, tag): counter
// (id, t, tag, block), four words per block.  Tag 0x20000 = initial
// injection, 0x10000 | k = k-th reinjection of the particle in a step.
struct Stream {
	uint32_t ctr[4];
	uint32_t buf[4];
	uint32_t key0, key1;
	int left;
	__device__ void init(uint64_t seed, uint32_t id, uint32_t t, uint32_t tag)
	{
		key0 = (uint32_t)seed;
		key1 = (uint32_t)(seed >> 32);
		ctr[0] = id;
		ctr[1] = t;
		ctr[2] = tag;
		ctr[3] = 0;
		left = 0;
	}
	__device__ uint32_t next()
	{
		if (left == 0) {
			buf[0] = ctr[0]; buf[1] = ctr[1]; buf[2] = ctr[2]; buf[3] = ctr[3];
			philox4x32(buf, key0, key1);
			ctr[3]++;
			left = 4;
		}
		return buf[4 - left--];
	}
	// rnd(state, maximum) of prng.c:11-28: maximum * u / UINT32_MAX.
	__device__ double rnd(double maximum) { return maximum * ((double)next() / 4294967295.0); }
};

// The grid a kernel body runs in.  A kernel of one run passes GridSelf (its
// own block index and grid size); a batched launch, which covers several
// member runs with one grid, passes each block its index and grid size
// within its member's share (GridSeg, from seg_block).
struct GridSelf {
	__device__ __forceinline__ uint32_t id() const { return blockIdx.x; }
	__device__ __forceinline__ uint32_t n() const { return gridDim.x; }
};
struct GridSeg {
	uint32_t i, c;
	__device__ __forceinline__ uint32_t id() const { return i; }
	__device__ __forceinline__ uint32_t n() const { return c; }
};

// Block `blockIdx.x` of a batched launch: its member m (pre[m] <= blockIdx.x
// < pre[m + 1], pre an exclusive prefix of the members' block counts) and
// its block index and grid size within that member's share of the launch.
struct SegBlock {
	uint32_t m, id, n;
};
__device__ __forceinline__ SegBlock seg_block(const uint32_t* __restrict__ pre, uint32_t M)
{
	uint32_t lo = 0, hi = M;  // pre[lo] <= b < pre[hi]
	const uint32_t b = blockIdx.x;
	while (hi - lo > 1) {
		const uint32_t mid = (lo + hi) >> 1;
		if (__ldg(&pre[mid]) <= b) lo = mid; else hi = mid;
	}
	const uint32_t p0 = __ldg(&pre[lo]);
	return SegBlock { lo, b - p0, __ldg(&pre[lo + 1]) - p0 };
}

__device__ __forceinline__ void set_status(RunRec* rec, int code)
{
	atomicCAS(&rec->status, 0, code);
}

__host__ __device__ inline int species_of_id(uint32_t id, uint32_t n_ions)
{
	return id == 0 ? SP_DUST : (id <= n_ions ? SP_ION : SP_E);
}

}  // namespace pot
