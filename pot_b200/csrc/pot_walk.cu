// Barnes-Hut walks fused with the Boris push, grain absorption and the
// boundary test; edge potential (chi_b); grain update.
//
// Plain form (POT_FORM_PLAIN): one thread per target, FP64, leaf size 1, the
// reference's stack discipline (children pushed in member order, popped
// last-first, pot.c:1755-1772), opening test and force expressions
// (pot.c:1719-1803) with unfused products so every accept/open decision is
// the reference's.  The reference accumulates in x87 long double; here the
// accumulation is FP64 with fused multiply-adds.
//
// Fast form (POT_FORM_FAST): see pot_walk_fast.cu.
#include "pot_push.cuh"

namespace pot {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// E (V/m) at (x, y, z) for the particle in Morton slot `self`:
// field_particle_feels_at, pot.c:1696-1808 (monopole cells).
// E[] holds the starting field on entry: zero, or a spheroidal grain's own
// field (pot-spheroid.c:1815-1819).
__device__ int field_plain(uint32_t self, double x, double y, double z, const TreeDev& T,
                           const double4* __restrict__ src64, const Params& P, double E[3],
                           uint32_t& n_inter)
{
	int32_t stack[WALK_STACK];
	int len = 1;
	stack[0] = 0;
	double ex = E[0], ey = E[1], ez = E[2];
	while (len) {
		const int32_t code = stack[--len];
		if (code >= 0) {
			const double4 c = T.cq[code];
			const double dx = dsub(x, c.x), dy = dsub(y, c.y), dz = dsub(z, c.z);
			const double dist2 = dsq3(dx, dy, dz);
			if (T.w2[code] < dmul(P.oap2, dist2)) {
				if (T.dip) {
					if (T.aq[code] != 0) {
						// DIPOLES, pot.c:1739-1745: the cell's dipole term too
						const double dist = sqrt(dist2);
						const double es = ddiv(QE, dmul(dmul(P.k4, dist2), dist));
						const double4 pd = T.dip[code];
						const double rp = ddiv(dadd(dadd(dmul(dx, pd.x), dmul(dy, pd.y)), dmul(dz, pd.z)), dist2);
						ex = fma(es, dadd(dsub(dmul(c.w, dx), pd.x), dmul(dmul(3.0, dx), rp)), ex);
						ey = fma(es, dadd(dsub(dmul(c.w, dy), pd.y), dmul(dmul(3.0, dy), rp)), ey);
						ez = fma(es, dadd(dsub(dmul(c.w, dz), pd.z), dmul(dmul(3.0, dz), rp)), ez);
						n_inter++;
					}
				} else if (c.w != 0.0) {
					const double dist = sqrt(dist2);
					const double es = dmul(ddiv(QE, dmul(dmul(P.k4, dist2), dist)), c.w);
					ex = fma(es, dx, ex);
					ey = fma(es, dy, ey);
					ez = fma(es, dz, ez);
					n_inter++;
				}
			} else {
				if (len + 8 > WALK_STACK) {
					E[0] = E[1] = E[2] = 0.0;
					return POT_E_WALK;
				}
				const int32_t* ch = &T.child[8u * (uint32_t)code];
#pragma unroll
				for (int s = 0; s < 8; s++) {
					const int32_t cc = ch[slot_digit(s)];
					if (cc != CH_EMPTY) stack[len++] = cc;
				}
			}
		} else {
			const uint32_t e = leaf_payload(code);
			uint32_t j0 = e, j1 = e + 1;
			if (e >= P.n_tree) {  // overflow bucket (see OVF_CAP)
				const uint2 r = T.ovf[e - P.n_tree];
				j0 = r.x;
				j1 = r.x + r.y;
			}
			for (uint32_t slot = j0; slot < j1; slot++) {
				if (slot == self) continue;
				const double4 p = src64[slot];
				const double dx = dsub(x, p.x), dy = dsub(y, p.y), dz = dsub(z, p.z);
				double dist2 = dsq3(dx, dy, dz);
				if (dist2 == 0.0) {
					E[0] = E[1] = E[2] = 0.0;
					return POT_E_COINCIDENT;
				}
				dist2 = dadd(dist2, P.soft2);
				const double dist = sqrt(dist2);
				const double es = ddiv(dmul(QE, p.w), dmul(dmul(P.k4, dist2), dist));
				ex = fma(es, dx, ex);
				ey = fma(es, dy, ey);
				ez = fma(es, dz, ez);
				n_inter++;
			}
		}
	}
	E[0] = ex;
	E[1] = ey;
	E[2] = ez;
	return POT_OK;
}

// phi_particle_feels (pot.c:1934-2018): potential at (x, y, z) for the
// particle in slot `self`, which is excluded; cells unsoftened, pairs
// softened, the reference's visit order and expressions.
__device__ double phi_plain(uint32_t self, double x, double y, double z, const TreeDev& T,
                            const double4* __restrict__ src64, const Params& P, int& rc)
{
	int32_t stack[WALK_STACK];
	int len = 1;
	stack[0] = 0;
	double phi = 0.0;
	while (len) {
		const int32_t code = stack[--len];
		if (code >= 0) {
			const double4 c = T.cq[code];
			const double dx = dsub(x, c.x), dy = dsub(y, c.y), dz = dsub(z, c.z);
			const double dist2 = dsq3(dx, dy, dz);
			if (T.w2[code] < dmul(P.oap2, dist2)) {
				if (T.dip) {
					if (T.aq[code] != 0) {  // DIPOLES, pot.c:1966-1974
						const double dist = sqrt(dist2);
						const double4 pd = T.dip[code];
						const double rp = dadd(dadd(dmul(dx, pd.x), dmul(dy, pd.y)), dmul(dz, pd.z));
						phi += ddiv(dmul(QE, dadd(ddiv(c.w, dist), ddiv(rp, dmul(dist, dist2)))), P.k4);
					}
				} else if (c.w != 0.0) {
					phi += ddiv(dmul(QE, c.w), dmul(P.k4, sqrt(dist2)));
				}
			} else {
				if (len + 8 > WALK_STACK) {
					rc = POT_E_WALK;
					return 0.0;
				}
				const int32_t* ch = &T.child[8u * (uint32_t)code];
#pragma unroll
				for (int s = 0; s < 8; s++) {
					const int32_t cc = ch[slot_digit(s)];
					if (cc != CH_EMPTY) stack[len++] = cc;
				}
			}
		} else {
			const uint32_t e = leaf_payload(code);
			uint32_t j0 = e, j1 = e + 1;
			if (P.leaf_size > 1 || e >= P.n_tree) {
				const uint2 r = P.leaf_size > 1 ? T.lrange[e] : T.ovf[e - P.n_tree];
				j0 = r.x;
				j1 = r.x + r.y;
			}
			for (uint32_t slot = j0; slot < j1; slot++) {
				if (slot == self) continue;
				const double4 p = src64[slot];
				const double d2 = dsq3(dsub(x, p.x), dsub(y, p.y), dsub(z, p.z));
				phi += ddiv(dmul(QE, p.w), dmul(P.k4, sqrt(dadd(d2, P.soft2))));
			}
		}
	}
	return phi;
}

// Deterministic block sum of three doubles (fixed shuffle and warp order).
__device__ void block_sum3(double v[3], double* __restrict__ out)
{
	__shared__ double part[32][3];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < 3; k++)
		for (int o = 16; o; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
	if (lane == 0)
		for (int k = 0; k < 3; k++) part[w][k] = v[k];
	__syncthreads();
	if (threadIdx.x == 0) {
		double t[3] = { 0.0, 0.0, 0.0 };
		for (int j = 0; j < (int)(blockDim.x >> 5); j++)
			for (int k = 0; k < 3; k++) t[k] += part[j][k];
		for (int k = 0; k < 3; k++) out[k] = t[k];
	}
}

// compute_epe of move_particles (pot.c:2771-2804), plain form: every
// particle's potential at its step-start position; per-block partial sums
// of q e phi per species (slots assigned to blocks statically).
__global__ void __launch_bounds__(128) k_epe_plain(const double4* __restrict__ pos, TreeDev T,
                                                   const double4* __restrict__ src64, double* __restrict__ partial,
                                                   Params P, RunRec* rec)
{
	double acc[3] = { 0.0, 0.0, 0.0 };
	if (rec->status == POT_OK) {
		const uint32_t gs = rec->grain_slot;
		for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.n; s += gridDim.x * blockDim.x) {
			const double4 p = src64[s];
			int rc = POT_OK;
			double phi = phi_plain(s, p.x, p.y, p.z, T, src64, P, rc);
			if (rc != POT_OK) set_status(rec, rc);
			if (s == gs) {
				rec->phi_grain = phi;
				continue;
			}
			if (P.shape) {  // pot-spheroid.c:2107-2109: the grain's own potential first
				phi = spheroid_phi(P, (double)rec->grain_q, dsub(p.x, rec->grain_pos[0]), dsub(p.y, rec->grain_pos[1]),
				                   dsub(p.z, rec->grain_pos[2])) + phi;
			}
			const int sp = (int)pos[s].w;
			acc[sp] += (QE * p.w) * phi;
		}
	}
	block_sum3(acc, &partial[3 * blockIdx.x]);
}

// Fixed-order sum of per-block (or per-group) partials into rec->epe.
__global__ void __launch_bounds__(1024) k_epe_final(const double* __restrict__ partial, const unsigned int* count,
                                                    uint32_t fixed, RunRec* rec)
{
	const uint32_t n = count ? *count : fixed;
	double v[3] = { 0.0, 0.0, 0.0 };
	for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
		for (int k = 0; k < 3; k++) v[k] += partial[3 * i + k];
	__shared__ double out[3];
	block_sum3(v, out);
	__syncthreads();
	if (threadIdx.x == 0) {
		rec->epe[SP_ION] = out[SP_ION];
		rec->epe[SP_E] = out[SP_E];
	}
}

__device__ __forceinline__ void warp_add_u64(unsigned long long* dst, unsigned long long v)
{
#pragma unroll
	for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	if (lane_id() == 0 && v) atomicAdd(dst, v);
}

// The walk fused with the push.  STG 0: Boris (half drift, field, kick,
// rotate, kick, half drift), then absorption and the boundary.  The
// non-Boris integrators take two launches: STG 1 evaluates the field at the
// old position and writes the intermediate state, its acceleration and its
// source entry (sb); STG 2 evaluates the field at the intermediate state over
// those sources (leaf particles moved, cells as built) and finishes the step
// (pot.c:2533-2639), then absorption and the boundary against the
// start-of-step position in src64.
template <int STG>
__global__ void __launch_bounds__(128) k_push_plain(double4* __restrict__ pos, double4* __restrict__ vel, TreeDev T,
                                                    const double4* __restrict__ src64,
                                                    const uint32_t* __restrict__ due_list,
                                                    uint32_t* __restrict__ rein_list, Params P, RunRec* rec,
                                                    StageBufs sb)
{
	if (rec->status != POT_OK) return;
	const uint32_t n_due = rec->n_due;
	const unsigned long long t = rec->t_steps;
	const bool grain_due = rec->grain_due != 0;
	const bool absorb_on = !(P.flags & FLAG_NO_GRAIN) && t >= P.t_settle;
	double gx = rec->grain_pos[0], gy = rec->grain_pos[1], gz = rec->grain_pos[2];
	if (STG == 2 && grain_due && rec->grain_slot < P.n) {
		const double4 g = pos[rec->grain_slot];  // the grain's intermediate position
		gx = g.x; gy = g.y; gz = g.z;
	}
	const double qg = (double)rec->grain_q;
	const double4* __restrict__ src = STG == 2 ? sb.src64b : src64;
	unsigned long long n_inter = 0, n_push = 0;
	for (;;) {
		uint32_t base = 0;
		if (lane_id() == 0) base = atomicAdd(&rec->work_ctr, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n_due) break;
		const uint32_t i = base + lane_id();
		if (i >= n_due) continue;
		const uint32_t s = due_list[i];
		const double4 p = pos[s];
		double4 v = vel[s];
		const int sp = (int)p.w;
		const double dt = P.dt * (double)P.tss[sp];
		const double half = 0.5 * dt;
		const double3 h = STG == 0 ? make_double3(fma(half, v.x, p.x), fma(half, v.y, p.y), fma(half, v.z, p.z))
		                           : make_double3(p.x, p.y, p.z);
		double E[3] = { 0.0, 0.0, 0.0 };
		if (P.shape && sp != SP_DUST) spheroid_field(P, qg, dsub(h.x, gx), dsub(h.y, gy), dsub(h.z, gz), E);
		uint32_t ni = 0;
		const int rc = field_plain(s, h.x, h.y, h.z, T, src, P, E, ni);
		if (rc != POT_OK) set_status(rec, rc);
		n_inter += ni;
		const double charge = sp == SP_DUST ? qg : (sp == SP_ION ? 1.0 : -1.0);
		const double qom = (QE * charge) / mass_of(sp, P);
		if (STG == 1) {
			const double3 a1 = accel_lorentz(E, v, qom, P);
			double4 pm = p;
			half_first(pm, v, a1, dt, P);
			pos[s] = pm;
			vel[s] = v;
			sb.acc[s] = make_double4(a1.x, a1.y, a1.z, 0.0);
			sb.src64b[s] = make_double4(pm.x, pm.y, pm.z, src64[s].w);
			continue;
		}
		n_push++;
		double3 xn;
		if (STG == 0) {
			boris(v, h, E, qom, dt, P, xn);
		} else {
			const double4 a = sb.acc[s];
			half_second(xn, v, p, make_double3(a.x, a.y, a.z), accel_lorentz(E, v, qom, P), dt, P);
		}
		uint32_t reason = 0;
		if (!grain_due) reason = after_push(sp, STG == 0 ? p : src64[s], xn, v, P, rec, absorb_on, gx, gy, gz);
		pos[s] = make_double4(xn.x, xn.y, xn.z, p.w);
		vel[s] = v;
		if (reason) rein_list[atomicAdd(&rec->n_rein, 1u)] = s | (reason << 30);
	}
	warp_add_u64(&rec->interactions, n_inter);
	warp_add_u64(&rec->n_pushed, n_push);
}

// Steps where the grain itself moves (t a multiple of tss[DUST]): the
// reference tests absorption against the grain's new position
// (new_parts[0], pot.c:2641-2652), so the tests run after all pushes.
template <class G>
__device__ __forceinline__ void absorb_late_body(G grd, double4* __restrict__ pos, double4* __restrict__ vel,
                                                 const double4* __restrict__ src64,
                                                 const uint32_t* __restrict__ due_list,
                                                 uint32_t* __restrict__ rein_list, const Params& P, RunRec* rec)
{
	if (rec->status != POT_OK || !rec->grain_due) return;
	const uint32_t n_due = rec->n_due;
	const bool absorb_on = !(P.flags & FLAG_NO_GRAIN) && rec->t_steps >= P.t_settle;
	const double4 g = pos[rec->grain_slot];
	for (uint32_t i = grd.id() * blockDim.x + threadIdx.x; i < n_due; i += grd.n() * blockDim.x) {
		const uint32_t s = due_list[i];
		const double4 p = pos[s];
		double4 v = vel[s];
		const double4 p_old = src64[s];
		const int sp = (int)p.w;
		double3 xn = make_double3(p.x, p.y, p.z);
		const uint32_t reason = after_push(sp, p_old, xn, v, P, rec, absorb_on, g.x, g.y, g.z);
		if (P.bounce > 0.0 && !reason) {  // a bounce moved it
			pos[s] = make_double4(xn.x, xn.y, xn.z, p.w);
			vel[s] = v;
		}
		if (reason) rein_list[atomicAdd(&rec->n_rein, 1u)] = s | (reason << 30);
	}
}

__global__ void k_absorb_late(double4* __restrict__ pos, double4* __restrict__ vel, const double4* __restrict__ src64,
                              const uint32_t* __restrict__ due_list, uint32_t* __restrict__ rein_list, Params P,
                              RunRec* rec)
{
	absorb_late_body(GridSelf {}, pos, vel, src64, due_list, rein_list, P, rec);
}

// Poisson variate by inversion (prng.c:50-70): walk the CDF from k = 0 until
// the uniform draw is used up.  The reference loops until the term
// underflows; the cap (the oracle's too) only ends a loop that cannot end
// (a rate of NaN or infinity), returning 0 as the reference's exit does.
constexpr uint32_t POISSON_CAP = 1u << 20;
__device__ uint32_t poisson_inv(double lambda, double uni, bool& capped)
{
	const double e = exp(-lambda);
	uint32_t k = 0;
	double ratio = 1.0;
	while (ratio != 0.0) {
		uni = dsub(uni, dmul(ratio, e));
		if (uni < 0.0) break;
		k++;
		ratio = dmul(ratio, ddiv(lambda, (double)k));
		if (k >= POISSON_CAP) {
			capped = true;
			return 0;
		}
	}
	return ratio != 0.0 ? k : 0;
}

// Grain update of pot.c:2825-2848 and the step's statistics.
template <class G>
__device__ __forceinline__ void grain_end_body(G grd, double4* __restrict__ pos, double4* __restrict__ vel,
                                               StepHist* hist, const Params& P, RunRec* rec, int epe)
{
	if (threadIdx.x != 0 || grd.id() != 0) return;
	const double dm = (double)rec->nabs_ion * P.m_ion + (double)rec->nabs_e * MASS_E;
	const double m = rec->grain_m + dm;
	double dp[3];
	for (int k = 0; k < 3; k++) {
		dp[k] = MASS_E * ((double)rec->sumv_e[k] / VFIX) + P.m_ion * ((double)rec->sumv_ion[k] / VFIX);
	}
	const uint32_t gs = rec->grain_slot;
	double gv[3] = { rec->grain_vel[0], rec->grain_vel[1], rec->grain_vel[2] };
	if (gs < P.n) {
		const double4 v = vel[gs];
		gv[0] = v.x; gv[1] = v.y; gv[2] = v.z;
	}
	for (int k = 0; k < 3; k++) gv[k] += dp[k] / m;
	if (gs < P.n) {
		vel[gs] = make_double4(gv[0], gv[1], gv[2], 0.0);
		if (rec->grain_due) {
			const double4 p = pos[gs];
			rec->grain_pos[0] = p.x; rec->grain_pos[1] = p.y; rec->grain_pos[2] = p.z;
		}
	}
	for (int k = 0; k < 3; k++) rec->grain_vel[k] = gv[k];
	rec->grain_m = m;
	rec->grain_q += rec->dq;
	if ((P.flags & FLAG_POIS) && rec->t_steps >= P.t_settle) {
		// POIS_POS_COLLECTION, pot.c:2837-2854: the OML ion flux at the cached
		// ion temperature and the grain's charge after this step's absorptions
		const double kb_ti = KB * rec->ion_temp;
		double phi_normed = dmul(dmul(QE, QE), (double)rec->grain_q);
		phi_normed = ddiv(phi_normed, dmul(dmul(dmul(4.0 * PI_REF, EPSILON0), P.a), kb_ti));
		const double lambda = dmul(dmul(P.pos_rate_const, sqrt(kb_ti)), dsub(1.0, phi_normed));
		Stream st;
		st.init(P.seed, 0u, (uint32_t)rec->t_steps, 0x30000u);
		bool capped = false;
		const uint32_t k = poisson_inv(lambda, st.rnd(1.0), capped);
		if (capped) rec->warn |= WARN_POISSON;
		rec->n_collected = k;
		rec->grain_q += k;
	}
	rec->q_sum += rec->grain_q;
	rec->tot_absor_e += rec->de;
	if (epe) {
		// the grain's energy with its updated charge, pot.c:2859-2864
		rec->epe[SP_DUST] = rec->grain_q ? (double)rec->grain_q * QE * rec->phi_grain : 0.0;
	}
	StepHist h;
	h.t_steps = rec->t_steps;
	h.grain_q = rec->grain_q;
	h.dq = rec->dq;
	h.de = rec->de;
	h.n_absorbed = rec->nabs_ion + rec->nabs_e;
	h.n_reinjected = rec->n_rein;
	h.n_pushed = rec->n_pushed;
	h.interactions = rec->interactions;
	h.far_cells = rec->far_cells;
	h.n_nodes = rec->n_nodes;
	h.chi_b = rec->chi_b;
	h.status = rec->status;
	h.pad = (int)rec->warn;
	for (int k = 0; k < 3; k++) h.epe[k] = epe ? rec->epe[k] : 0.0;
	hist[rec->t_steps % HIST] = h;
}

__global__ void k_grain_end(double4* __restrict__ pos, double4* __restrict__ vel, StepHist* hist, Params P,
                            RunRec* rec, int epe)
{
	grain_end_body(GridSelf {}, pos, vel, hist, P, rec, epe);
}

// ---------------------------------------------------------------------------
// potential: warp-cooperative phi_at (pot.c:1818-1901)
// ---------------------------------------------------------------------------
constexpr int PHI_STACK = 2048;

// One warp evaluates the potential at (x, y, z); `stack` is this warp's
// shared-memory stack.  Nodes are processed 32 at a time; children of opened
// cells are pushed with a warp prefix sum.  Returns NaN on stack overflow.
__device__ double warp_phi(double x, double y, double z, const TreeDev& T, const double4* __restrict__ src64,
                           const Params& P, int32_t* stack)
{
	const uint32_t lane = lane_id();
	int len = 1;
	if (lane == 0) stack[0] = 0;
	__syncwarp();
	double acc = 0.0;
	bool overflow = false;
	while (len > 0) {
		const int take = len < 32 ? len : 32;
		const int32_t code = (int)lane < take ? stack[len - 1 - (int)lane] : CH_EMPTY;
		__syncwarp();
		len -= take;
		int32_t ch[8];
		int nch = 0;
		if (code >= 0) {
			const double4 c = T.cq[code];
			const double dx = dsub(x, c.x), dy = dsub(y, c.y), dz = dsub(z, c.z);
			const double dist2 = dsq3(dx, dy, dz);
			if (T.w2[code] < dmul(P.oap2, dist2)) {
				if (T.dip) {
					if (T.aq[code] != 0) {  // DIPOLES, pot.c:1860-1868
						const double dist = sqrt(dist2);
						const double4 pd = T.dip[code];
						const double rp = dadd(dadd(dmul(dx, pd.x), dmul(dy, pd.y)), dmul(dz, pd.z));
						acc += dmul(ddiv(QE, P.k4), dadd(ddiv(c.w, dist), ddiv(rp, dmul(dist, dist2))));
					}
				} else if (c.w != 0.0) {
					acc += ddiv(dmul(QE, c.w), dmul(P.k4, sqrt(dist2)));
				}
			} else {
				const int32_t* cp = &T.child[8u * (uint32_t)code];
#pragma unroll
				for (int s = 0; s < 8; s++) {
					const int32_t cc = cp[slot_digit(s)];
					if (cc != CH_EMPTY) ch[nch++] = cc;
				}
			}
		} else if (code != CH_EMPTY) {
			const uint32_t e = leaf_payload(code);
			uint32_t j0 = e, j1 = e + 1;
			if (P.leaf_size > 1 || e >= P.n_tree) {
				const uint2 r = P.leaf_size > 1 ? T.lrange[e] : T.ovf[e - P.n_tree];
				j0 = r.x;
				j1 = r.x + r.y;
			}
			for (uint32_t j = j0; j < j1; j++) {
				const double4 p = src64[j];
				const double d2 = dsq3(dsub(x, p.x), dsub(y, p.y), dsub(z, p.z));
				acc += ddiv(dmul(QE, p.w), dmul(P.k4, sqrt(dadd(d2, P.soft2))));
			}
		}
		int incl = nch;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int tv = __shfl_up_sync(0xffffffffu, incl, o);
			if ((int)lane >= o) incl += tv;
		}
		const int total = __shfl_sync(0xffffffffu, incl, 31);
		if (len + total > PHI_STACK) {
			overflow = true;
			break;
		}
		const int off = len + incl - nch;
		for (int j = 0; j < nch; j++) stack[off + j] = ch[j];
		__syncwarp();
		len += total;
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
	return overflow ? __longlong_as_double(0x7ff8000000000000ll) : acc;
}

// The spheroid's term of phi_at (pot-spheroid.c:1924-1953), which the
// reference evaluates at the point's own coordinates rather than relative
// to the grain; reproduced as written.  Zero for a spherical grain, whose
// charge is a tree source.
__device__ __forceinline__ double spheroid_phi_at(const Params& P, const RunRec* rec, double x, double y, double z)
{
	if (!P.shape) return 0.0;
	double u, v, w;
	sph_to_frame(P, x, y, z, u, v, w);
	return spheroid_phi_frame(P, (double)rec->grain_q, u, v, w);
}

// measure_chi_b (pot.c:2251-2279) as a run of P = chi_ranks MPI ranks does
// it (pot.c:2409-2418): rank k samples phi at azimuth 2 pi k / P in the x-y
// plane through the grain, the samples are summed and divided by P; every 20
// steps.  Four warps share the samples; the sum is taken in rank order.
template <class G>
__device__ __forceinline__ void chi_b_body(G grd, const TreeDev& T, const double4* __restrict__ src64,
                                           const Params& P, RunRec* rec, int force)
{
	__shared__ int32_t stack[4][PHI_STACK];
	__shared__ double sample[64];
	__shared__ int bad;
	if (!(P.flags & FLAG_SCEPTIC) || rec->status != POT_OK) return;
	if (!force && (rec->t_steps % 20) != 0) return;
	const uint32_t w = threadIdx.x >> 5;
	if (threadIdx.x == 0) bad = 0;
	__syncthreads();
	const double zen = PI_REF / 2.0;
	const double r = P.rad;
	for (uint32_t k = w; k < P.chi_ranks; k += 4) {
		const double azi = 2.0 * PI_REF * k / P.chi_ranks;
		const double x = rec->grain_pos[0] + (r * cos(azi) * sin(zen));
		const double y = rec->grain_pos[1] + (r * sin(azi) * sin(zen));
		const double z = rec->grain_pos[2] + (r * cos(zen));
		const double phi = spheroid_phi_at(P, rec, x, y, z) + warp_phi(x, y, z, T, src64, P, stack[w]);
		if (lane_id() == 0) {
			sample[k] = phi / (KB * P.Ti / (1 * QE));
			if (isnan(phi)) bad = 1;
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		if (bad) {
			set_status(rec, POT_E_WALK);
		} else {
			double sum = 0.0;
			for (uint32_t k = 0; k < P.chi_ranks; k++) sum += sample[k];
			rec->chi_b = sum / P.chi_ranks;
		}
	}
}

__global__ void __launch_bounds__(128) k_chi_b(TreeDev T, const double4* __restrict__ src64, Params P, RunRec* rec,
                                               int force)
{
	chi_b_body(GridSelf {}, T, src64, P, rec, force);
}

__global__ void k_phi_query(TreeDev T, const double4* __restrict__ src64, const double* __restrict__ xyz,
                            uint32_t nq, double* __restrict__ phi, Params P, RunRec* rec)
{
	__shared__ int32_t stack[4][PHI_STACK];
	const uint32_t w = threadIdx.x >> 5;
	for (uint32_t q = blockIdx.x * 4 + w; q < nq; q += gridDim.x * 4) {
		const double v = spheroid_phi_at(P, rec, xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]) +
		                 warp_phi(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2], T, src64, P, stack[w]);
		if (lane_id() == 0) {
			phi[q] = v;
			if (isnan(v)) set_status(rec, POT_E_WALK);
		}
	}
}

__global__ void k_field_query_plain(TreeDev T, const double4* __restrict__ src64, const double* __restrict__ xyz,
                                    const uint32_t* __restrict__ self_slot, uint32_t nq, double* __restrict__ E,
                                    Params P, RunRec* rec)
{
	const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= nq) return;
	double e[3] = { 0.0, 0.0, 0.0 };
	if (P.shape && self_slot[q] != rec->grain_slot) {
		spheroid_field(P, (double)rec->grain_q, dsub(xyz[3 * q], rec->grain_pos[0]), dsub(xyz[3 * q + 1], rec->grain_pos[1]),
		               dsub(xyz[3 * q + 2], rec->grain_pos[2]), e);
	}
	uint32_t ni = 0;
	const int rc = field_plain(self_slot[q], xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2], T, src64, P, e, ni);
	if (rc != POT_OK) set_status(rec, rc);
	E[3 * q] = e[0];
	E[3 * q + 1] = e[1];
	E[3 * q + 2] = e[2];
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
void launch_push_fast(double4* pos, double4* vel, const TreeDev& T, const float4* src32, const double4* src64,
                      const uint32_t* due_list, const uint2* groups, uint32_t* rein_list, const Params& P,
                      RunRec* rec, const StageBufs& sb, cudaStream_t s, Timer& tm);
void launch_epe_fast(const double4* pos, const TreeDev& T, const float4* src32, const double4* src64,
                     uint2* groups_all, double* partial, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);
void launch_field_query_fast(const TreeDev& T, const float4* src32, const double* xyz, const uint32_t* self_slot,
                             uint32_t nq, double* E, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);

static int sm_count()
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

void launch_chi_b(const TreeDev& T, const double4* src64, const Params& P, RunRec* rec, int force,
                  cudaStream_t s, Timer& tm)
{
	if (!(P.flags & FLAG_SCEPTIC)) return;
	ScopedKernel k(tm, "chi_b");
	k_chi_b<<<1, 128, 0, s>>>(T, src64, P, rec, force);
}

void launch_push(double4* pos, double4* vel, const TreeDev& T, const double4* src64, const float4* src32,
                 const uint32_t* due_list, const uint2* groups, uint32_t* rein_list, const Params& P, RunRec* rec,
                 const StageBufs& sb, cudaStream_t s, Timer& tm)
{
	if (P.form == POT_FORM_FAST) {
		launch_push_fast(pos, vel, T, src32, src64, due_list, groups, rein_list, P, rec, sb, s, tm);
		return;
	}
	ScopedKernel k(tm, sb.stage == 0 ? "walk_push_plain" : (sb.stage == 1 ? "walk_half1_plain" : "walk_half2_plain"));
	const int nb = sm_count() * 8;
	if (sb.stage == 0) {
		k_push_plain<0><<<nb, 128, 0, s>>>(pos, vel, T, src64, due_list, rein_list, P, rec, sb);
	} else if (sb.stage == 1) {
		k_push_plain<1><<<nb, 128, 0, s>>>(pos, vel, T, src64, due_list, rein_list, P, rec, sb);
	} else {
		k_push_plain<2><<<nb, 128, 0, s>>>(pos, vel, T, src64, due_list, rein_list, P, rec, sb);
	}
}

void launch_absorb_late(double4* pos, double4* vel, const double4* src64, const uint32_t* due_list,
                        uint32_t* rein_list, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "absorb_late");
	k_absorb_late<<<sm_count(), 256, 0, s>>>(pos, vel, src64, due_list, rein_list, P, rec);
}

void launch_grain_end(double4* pos, double4* vel, StepHist* hist, const Params& P, RunRec* rec, int epe,
                      cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "grain_end");
	k_grain_end<<<1, 32, 0, s>>>(pos, vel, hist, P, rec, epe);
}

void launch_epe(const double4* pos, const TreeDev& T, const double4* src64, const float4* src32, uint2* groups_all,
                double* partial, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	if (P.form == POT_FORM_FAST) {
		launch_epe_fast(pos, T, src32, src64, groups_all, partial, P, rec, s, tm);
		ScopedKernel k(tm, "epe_final");
		k_epe_final<<<1, 1024, 0, s>>>(partial, &rec->n_groups_all, 0, rec);
		return;
	}
	ScopedKernel k(tm, "epe_plain", 2);
	k_epe_plain<<<EPE_BLOCKS, 128, 0, s>>>(pos, T, src64, partial, P, rec);
	k_epe_final<<<1, 1024, 0, s>>>(partial, nullptr, EPE_BLOCKS, rec);
}

void launch_field_query(const TreeDev& T, const double4* src64, const float4* src32, const double* xyz,
                        const uint32_t* self_slot, uint32_t nq, double* E, const Params& P, RunRec* rec,
                        cudaStream_t s, Timer& tm)
{
	if (P.form == POT_FORM_FAST) {
		launch_field_query_fast(T, src32, xyz, self_slot, nq, E, P, rec, s, tm);
		return;
	}
	ScopedKernel k(tm, "field_query");
	k_field_query_plain<<<(nq + 127) / 128, 128, 0, s>>>(T, src64, xyz, self_slot, nq, E, P, rec);
}

void launch_phi_query(const TreeDev& T, const double4* src64, const double* xyz, uint32_t nq, double* phi,
                      const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "phi_query");
	const uint32_t nb = (nq + 3) / 4;
	k_phi_query<<<nb < 4096 ? nb : 4096, 128, 0, s>>>(T, src64, xyz, nq, phi, P, rec);
}

}  // namespace pot

// ---------------------------------------------------------------------------
// packed batch: chi_b, late absorption and the grain update of every member
// ---------------------------------------------------------------------------
namespace pot {

__global__ void __launch_bounds__(128) kp_chi_b(PackDev B)
{
	const SegBlock sb = seg_block(B.pre[PS_ONE], B.M);
	const MemberView& v = B.mv[sb.m];
	chi_b_body(GridSeg { sb.id, sb.n }, v.T, v.src64, v.P, v.rec, 0);
}

__global__ void kp_absorb_late(PackDev B, int k)
{
	const SegBlock sb = seg_block(B.pre[PS_SMALL], B.M);
	const MemberView& v = B.mv[sb.m];
	const uint32_t b = pack_out(v, k);
	absorb_late_body(GridSeg { sb.id, sb.n }, v.pos[b], v.vel[b], v.src64, v.due_list, v.rein_list, v.P, v.rec);
}

__global__ void kp_grain_end(PackDev B, int k)
{
	const SegBlock sb = seg_block(B.pre[PS_ONE], B.M);
	const MemberView& v = B.mv[sb.m];
	const uint32_t b = pack_out(v, k);
	grain_end_body(GridSeg { sb.id, sb.n }, v.pos[b], v.vel[b], v.hist, v.P, v.rec, 0);
}

void pack_chi_b(const PackDev& B, cudaStream_t s)
{
	kp_chi_b<<<B.blocks[PS_ONE], 128, 0, s>>>(B);
}

void pack_absorb_late(const PackDev& B, int k, cudaStream_t s)
{
	kp_absorb_late<<<B.blocks[PS_SMALL], 256, 0, s>>>(B, k);
}

void pack_grain_end(const PackDev& B, int k, cudaStream_t s)
{
	kp_grain_end<<<B.blocks[PS_ONE], 32, 0, s>>>(B, k);
}

}  // namespace pot
