// Per-particle push, absorption and boundary helpers shared by the plain
// and fast walk kernels.
#pragma once

#include "pot_tree.cuh"

namespace pot {

// does_particle_cross_grain, pot.c:2287-2325, unfused.
__device__ __forceinline__ bool cross_grain(double px, double py, double pz, double dx, double dy, double dz,
                                            double gx, double gy, double gz, double a)
{
	const double s0 = dsub(gx, px), s1 = dsub(gy, py), s2 = dsub(gz, pz);
	const double ss = dsq3(s0, s1, s2);
	const double a2 = dmul(a, a);
	if (ss <= a2) return true;
	const double d2 = dsq3(dx, dy, dz);
	const double ds = dadd(dadd(dmul(dx, s0), dmul(dy, s1)), dmul(dz, s2));
	const double alpha = ddiv(ds, d2);
	if ((alpha < -1.0) || (alpha > 0.0)) return false;
	return dsub(ss, dmul(alpha, ds)) <= a2;
}

// check_particle_in_sim_area, pot.c:2071-2076 (spherical domain)
__device__ __forceinline__ bool outside_domain(double x, double y, double z, const Params& P)
{
	return sqrt(dsq3(dsub(x, P.rad), dsub(y, P.rad), dsub(z, P.rad))) > P.rad;
}

__device__ __forceinline__ double mass_of(int sp) { return sp == SP_DUST ? MASS_DUST : (sp == SP_ION ? MASS_ION : MASS_E); }

// Boris step of pot.c:2475-2532 given E at the half-drifted position h:
// v += dt a; rotate about b by 2 atan(dt qom |B| / 2); v += dt a;
// x = h + dt v / 2, with a = qom E / 2.
__device__ __forceinline__ void boris(double4& v, double3 h, const double E[3], double qom, double dt,
                                      const Params& P, double3& xn)
{
	const double ax = 0.5 * qom * E[0], ay = 0.5 * qom * E[1], az = 0.5 * qom * E[2];
	double vx = fma(dt, ax, v.x), vy = fma(dt, ay, v.y), vz = fma(dt, az, v.z);
	if (P.Bmag != 0.0) {
		const double dephi = 2.0 * atan(0.5 * dt * qom * P.Bmag);
		double sn, cs;
		sincos(dephi, &sn, &cs);
		const double* d = P.bhat;
		const double omc = 1.0 - cs;
		const double dot = d[0] * vx + d[1] * vy + d[2] * vz;
		const double t0 = d[0] * dot * omc + (vx * cs + (d[1] * vz - d[2] * vy) * sn);
		const double t1 = d[1] * dot * omc + (vy * cs + (d[2] * vx - d[0] * vz) * sn);
		const double t2 = d[2] * dot * omc + (vz * cs + (d[0] * vy - d[1] * vx) * sn);
		vx = t0; vy = t1; vz = t2;
	}
	vx = fma(dt, ax, vx);
	vy = fma(dt, ay, vy);
	vz = fma(dt, az, vz);
	const double half = 0.5 * dt;
	xn = make_double3(fma(half, vx, h.x), fma(half, vy, h.y), fma(half, vz, h.z));
	v = make_double4(vx, vy, vz, 0.0);
}

// Absorption tally (pot.c:2646-2666) for one absorbed particle.
__device__ __forceinline__ void tally_absorbed(RunRec* rec, int sp, const double4& v)
{
	if (sp == SP_E) {
		atomicAdd(&rec->de, 1ull);
		atomicAdd(&rec->nabs_e, 1ull);
		atomicAdd((unsigned long long*)&rec->dq, (unsigned long long)(long long)-1);
		atomicAdd((unsigned long long*)&rec->sumv_e[0], (unsigned long long)llrint(v.x * VFIX));
		atomicAdd((unsigned long long*)&rec->sumv_e[1], (unsigned long long)llrint(v.y * VFIX));
		atomicAdd((unsigned long long*)&rec->sumv_e[2], (unsigned long long)llrint(v.z * VFIX));
	} else {
		atomicAdd(&rec->nabs_ion, 1ull);
		atomicAdd((unsigned long long*)&rec->dq, 1ull);
		atomicAdd((unsigned long long*)&rec->sumv_ion[0], (unsigned long long)llrint(v.x * VFIX));
		atomicAdd((unsigned long long*)&rec->sumv_ion[1], (unsigned long long)llrint(v.y * VFIX));
		atomicAdd((unsigned long long*)&rec->sumv_ion[2], (unsigned long long)llrint(v.z * VFIX));
	}
}

// After the push: absorption (then reinjection, whose result is re-tested
// against the boundary by the reinjection kernel), else the boundary test.
// Returns the reinjection reason bits (1 absorbed, 2 outside).
__device__ __forceinline__ uint32_t after_push(int sp, const double4& p_old, const double3& xn, const double4& vn,
                                               const Params& P, RunRec* rec, bool absorb_on, double gx,
                                               double gy, double gz)
{
	uint32_t reason = 0;
	if (absorb_on && sp != SP_DUST &&
	    cross_grain(xn.x, xn.y, xn.z, dsub(xn.x, p_old.x), dsub(xn.y, p_old.y), dsub(xn.z, p_old.z), gx, gy, gz,
	                P.a)) {
		tally_absorbed(rec, sp, vn);
		reason = 1;
	} else if (outside_domain(xn.x, xn.y, xn.z, P)) {
		reason = 2;
	}
	return reason;
}

}  // namespace pot
