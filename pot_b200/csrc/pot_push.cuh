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

// ---- spheroidal grain (pot-spheroid.c, PROLATE / OBLATE programs) -------
// Grain-relative vectors are taken into the spheroid's frame (axis, e1, e2);
// for the reference's x axis that is the identity, bit for bit.  Products
// and sums are unfused and in the reference's order; the transcendental
// functions are CUDA's (within a few ulp of the host libm).

__device__ __forceinline__ void sph_to_frame(const Params& P, double dx, double dy, double dz, double& u, double& v,
                                             double& w)
{
	if (!P.s_tilted) {
		u = dx;
		v = dy;
		w = dz;
		return;
	}
	u = dadd(dadd(dmul(dx, P.s_ax[0]), dmul(dy, P.s_ax[1])), dmul(dz, P.s_ax[2]));
	v = dadd(dadd(dmul(dx, P.s_e1[0]), dmul(dy, P.s_e1[1])), dmul(dz, P.s_e1[2]));
	w = dadd(dadd(dmul(dx, P.s_e2[0]), dmul(dy, P.s_e2[1])), dmul(dz, P.s_e2[2]));
}

__device__ __forceinline__ void sph_from_frame(const Params& P, double u, double v, double w, double out[3])
{
	if (!P.s_tilted) {
		out[0] = u;
		out[1] = v;
		out[2] = w;
		return;
	}
#pragma unroll
	for (int k = 0; k < 3; k++) out[k] = dadd(dadd(dmul(u, P.s_ax[k]), dmul(v, P.s_e1[k])), dmul(w, P.s_e2[k]));
}

// rt of the prolate / oblate forms (pot-spheroid.c:1740-1752):
// rho2^2 + x^4 + c^4 + 2 rho2 x^2 -/+ 2 rho2 c^2 +/- 2 x^2 c^2, left to right
__device__ __forceinline__ double sph_rt(int shape, double rho2, double x, double fc)
{
	const double x4 = dmul(dmul(dmul(x, x), x), x);
	const double c4 = dmul(dmul(dmul(fc, fc), fc), fc);
	const double t4 = dmul(dmul(dmul(2.0, rho2), x), x);
	const double t5 = dmul(dmul(dmul(2.0, rho2), fc), fc);
	const double t6 = dmul(dmul(dmul(2.0, x), x), fc);
	const double t6c = dmul(t6, fc);
	const double head = dadd(dadd(dadd(dmul(rho2, rho2), x4), c4), t4);
	return shape == 1 ? sqrt(dsub(dadd(head, t5), t6c)) : sqrt(dadd(dsub(head, t5), t6c));
}

// field_particle_feels_from_grain (pot-spheroid.c:1689-1779) at
// grain-relative (dx, dy, dz) for grain charge q (elementary charges), V/m.
__device__ __forceinline__ void spheroid_field(const Params& P, double q, double dx, double dy, double dz,
                                               double E[3])
{
	double x, y, z;
	sph_to_frame(P, dx, dy, dz, x, y, z);
	const double fc = P.s_fc_f;
	const double phi_const = ddiv(dmul(dmul(QE, q), P.s_num), P.s_den_f);
	const double rho2 = dadd(dmul(y, y), dmul(z, z));
	const double rt = sph_rt((int)P.shape, rho2, x, fc);
	const double c2 = dmul(fc, fc);
	const double num = P.shape == 1 ? dadd(dsub(dadd(rho2, dmul(x, x)), c2), rt)
	                                : dadd(dadd(dadd(rho2, dmul(x, x)), c2), rt);
	const double e2 = ddiv(num, dmul(dmul(2.0, fc), fc));  // sinh^2 (prolate), cosh^2 (oblate)
	const double En = ddiv(-phi_const, sqrt(dmul(e2, rt)));
	const double beta = atan(ddiv(dmul(-e2, x), dmul(P.shape == 1 ? dadd(e2, 1.0) : dsub(e2, 1.0), sqrt(rho2))));
	const double theta = atan(ddiv(fabs(z), fabs(y)));
	const double cb = cos(beta);
	const double u = dmul(-En, sin(beta));
	const double v = ddiv(dmul(dmul(dmul(En, cb), cos(theta)), fabs(y)), y);
	const double w = ddiv(dmul(dmul(dmul(En, cb), sin(theta)), fabs(z)), z);
	sph_from_frame(P, u, v, w, E);
}

// the spheroid's potential at (x, y, z) already in its frame, V
// (pot-spheroid.c:2054-2078; the same forms at 1924-1953)
__device__ __forceinline__ double spheroid_phi_frame(const Params& P, double q, double x, double y, double z)
{
	const double fc = P.s_fc_p;
	const double phi_const = ddiv(dmul(dmul(QE, q), P.s_num), P.s_den_p);
	const double rho2 = dadd(dmul(y, y), dmul(z, z));
	const double rt = sph_rt((int)P.shape, rho2, x, fc);
	const double c2 = dmul(fc, fc);
	const double rx = dadd(rho2, dmul(x, x));
	const double ratio = ddiv(dsub(sqrt(dadd(dadd(rx, c2), rt)), dmul(fc, sqrt(2.0))), sqrt(dadd(dsub(rx, c2), rt)));
	return P.shape == 1 ? dmul(phi_const, log(ratio)) : dmul(phi_const, dsub(atan(ratio), dmul(0.25, PI_REF)));
}

// phi_particle_feels_from_grain: grain-relative (dx, dy, dz)
__device__ __forceinline__ double spheroid_phi(const Params& P, double q, double dx, double dy, double dz)
{
	double x, y, z;
	sph_to_frame(P, dx, dy, dz, x, y, z);
	return spheroid_phi_frame(P, q, x, y, z);
}

// does_particle_cross_grain of pot-spheroid.c:2448-2537, p the new position,
// d the step's displacement, g the grain.
__device__ __forceinline__ bool cross_spheroid(const Params& P, double px, double py, double pz, double ddx,
                                               double ddy, double ddz, double gx, double gy, double gz)
{
	double s0, s1, s2, d0, d1, d2;
	sph_to_frame(P, dsub(gx, px), dsub(gy, py), dsub(gz, pz), s0, s1, s2);
	sph_to_frame(P, ddx, ddy, ddz, d0, d1, d2);
	const double A = P.s_A;
	if (dadd(dmul(s0, s0), dmul(dmul(dadd(dmul(s1, s1), dmul(s2, s2)), A), A)) <= P.s_thr) return true;
	const double xm = ddiv(dadd(dmul(d1, dsub(dmul(d1, s0), dmul(d0, s1))), dmul(d2, dsub(dmul(d2, s0), dmul(d0, s2)))),
	                       dadd(dadd(ddiv(dmul(d0, d0), dmul(A, A)), dmul(d1, d1)), dmul(d2, d2)));
	const double xp = dsub(s0, d0);
	if (((xm > s0) && (xm > xp)) || ((xm < s0) && (xm < xp))) return false;
	const double ym = dadd(ddiv(dmul(d1, dsub(xm, s0)), d0), s1);
	const double zm = dadd(ddiv(dmul(d2, dsub(xm, s0)), d0), s2);
	return dadd(dmul(xm, xm), dmul(dmul(dadd(dmul(ym, ym), dmul(zm, zm)), A), A)) <= P.s_thr;
}

// check_particle_in_sim_area, pot.c:2071-2076 (spherical domain)
__device__ __forceinline__ bool outside_domain(double x, double y, double z, const Params& P)
{
	return sqrt(dsq3(dsub(x, P.rad), dsub(y, P.rad), dsub(z, P.rad))) > P.rad;
}

__device__ __forceinline__ double mass_of(int sp, const Params& P)
{
	return sp == SP_DUST ? MASS_DUST : (sp == SP_ION ? P.m_ion : MASS_E);
}

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

// Non-Boris integrators (pot.c:2533-2639), velocity Verlet and
// Euler-Richardson: the acceleration a = q/m (E + v x B) at the old state,
// then again at an intermediate state.
__device__ __forceinline__ double3 accel_lorentz(const double E[3], const double4& v, double qom, const Params& P)
{
	return make_double3(qom * dsub(dadd(E[0], dmul(v.y, P.B[2])), dmul(v.z, P.B[1])),
	                    qom * dsub(dadd(E[1], dmul(v.z, P.B[0])), dmul(v.x, P.B[2])),
	                    qom * dsub(dadd(E[2], dmul(v.x, P.B[1])), dmul(v.y, P.B[0])));
}

// First half (pot.c:2536-2551): v += dt/2 a1; x += dt/2 v0 (Euler-Richardson)
// or x += dt (v0 + dt/2 a1) (velocity Verlet).
__device__ __forceinline__ void half_first(double4& p, double4& v, const double3& a1, double dt, const Params& P)
{
	const double hd = 0.5 * dt;
	const double4 v0 = v;
	v.x = dadd(v0.x, dmul(hd, a1.x));
	v.y = dadd(v0.y, dmul(hd, a1.y));
	v.z = dadd(v0.z, dmul(hd, a1.z));
	if (P.integrator == POT_INT_EULER_RICHARDSON) {
		p.x = dadd(p.x, dmul(hd, v0.x));
		p.y = dadd(p.y, dmul(hd, v0.y));
		p.z = dadd(p.z, dmul(hd, v0.z));
	} else {
		p.x = dadd(p.x, dmul(dt, dadd(v0.x, dmul(hd, a1.x))));
		p.y = dadd(p.y, dmul(dt, dadd(v0.y, dmul(hd, a1.y))));
		p.z = dadd(p.z, dmul(dt, dadd(v0.z, dmul(hd, a1.z))));
	}
}

// Second half (pot.c:2624-2636) from the intermediate state (p, v): the
// Euler-Richardson position and velocity in the reference's round-trip form,
// or the velocity Verlet kick v += dt/2 a2.
__device__ __forceinline__ void half_second(double3& xn, double4& v, const double4& p, const double3& a1,
                                            const double3& a2, double dt, const Params& P)
{
	const double hd = 0.5 * dt;
	xn = make_double3(p.x, p.y, p.z);
	if (P.integrator == POT_INT_EULER_RICHARDSON) {
		const double4 vm = v;
		xn.x = dadd(dsub(p.x, dmul(hd, dsub(vm.x, dmul(hd, a1.x)))), dmul(dt, vm.x));
		xn.y = dadd(dsub(p.y, dmul(hd, dsub(vm.y, dmul(hd, a1.y)))), dmul(dt, vm.y));
		xn.z = dadd(dsub(p.z, dmul(hd, dsub(vm.z, dmul(hd, a1.z)))), dmul(dt, vm.z));
		v.x = dadd(dsub(vm.x, dmul(hd, a1.x)), dmul(dt, a2.x));
		v.y = dadd(dsub(vm.y, dmul(hd, a1.y)), dmul(dt, a2.y));
		v.z = dadd(dsub(vm.z, dmul(hd, a1.z)), dmul(dt, a2.z));
	} else {
		v.x = dadd(v.x, dmul(hd, a2.x));
		v.y = dadd(v.y, dmul(hd, a2.y));
		v.z = dadd(v.z, dmul(hd, a2.z));
	}
}

// OUT_BOUNCE at the spherical wall (pot.c:2036-2069): a particle outside the
// sphere and moving outwards has its radial velocity reversed, every
// spherical component scaled by the coefficient of restitution, and goes back
// to its start-of-step position; one moving inwards stays where it is (the
// reference's warning, pot.c:2719-2722).  Returns 0 inside, 1 bounced, 2 left
// in the wall.  The angles come from atan2 and acos in FP64 (atan2l and acosl,
// rounded to double, in the reference).
__device__ __forceinline__ int bounce_wall(const double4& p_old, double3& xn, double4& vn, const Params& P)
{
	const double dx = dsub(xn.x, P.rad), dy = dsub(xn.y, P.rad), dz = dsub(xn.z, P.rad);
	const double r0 = sqrt(dsq3(dx, dy, dz));
	if (!(r0 > P.rad)) return 0;
	const double ph = atan2(dy, dx);
	const double th = acos(ddiv(dz, r0));
	const double cp = cos(ph), sp = sin(ph), ct = cos(th), st = sin(th);
	double v0 = dadd(dadd(dmul(dmul(vn.x, cp), st), dmul(dmul(vn.y, sp), st)), dmul(vn.z, ct));
	double v1 = dadd(dmul(-vn.x, sp), dmul(vn.y, cp));
	double v2 = dsub(dadd(dmul(dmul(vn.x, cp), ct), dmul(dmul(vn.y, sp), ct)), dmul(vn.z, st));
	if (!(v0 > 0.0)) return 2;
	v0 = dmul(v0, -P.bounce);
	v1 = dmul(v1, P.bounce);
	v2 = dmul(v2, P.bounce);
	// velocity_in_cartesian_coords, coord.c:6-13
	vn.x = dadd(dsub(dmul(dmul(v0, cp), st), dmul(v1, sp)), dmul(dmul(v2, cp), ct));
	vn.y = dadd(dadd(dmul(dmul(v0, sp), st), dmul(v1, cp)), dmul(dmul(v2, sp), ct));
	vn.z = dsub(dmul(v0, ct), dmul(v2, st));
	xn = make_double3(p_old.x, p_old.y, p_old.z);
	return 1;
}

__device__ __forceinline__ void count_wall(RunRec* rec, int b)
{
	if (b == 1) {
		atomicAdd(&rec->n_bounced, 1u);
	} else if (b == 2) {
		atomicAdd(&rec->n_wall, 1u);
		atomicOr(&rec->warn, WARN_WALL);
	}
}

// Absorption tally (pot.c:2646-2666) for one absorbed particle.  With the
// Poisson ion collection an absorbed ion adds no charge (pot.c:2664-2670).
__device__ __forceinline__ void tally_absorbed(RunRec* rec, int sp, const double4& v, const Params& P)
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
		if (!(P.flags & FLAG_POIS)) atomicAdd((unsigned long long*)&rec->dq, 1ull);
		atomicAdd((unsigned long long*)&rec->sumv_ion[0], (unsigned long long)llrint(v.x * VFIX));
		atomicAdd((unsigned long long*)&rec->sumv_ion[1], (unsigned long long)llrint(v.y * VFIX));
		atomicAdd((unsigned long long*)&rec->sumv_ion[2], (unsigned long long)llrint(v.z * VFIX));
	}
}

// After the push: absorption (then reinjection, whose result is re-tested
// against the boundary by the reinjection kernel), else the boundary test:
// reinjection, or with OUT_BOUNCE the wall's bounce applied to (xn, vn) in
// place.  Returns the reinjection reason bits (1 absorbed, 2 outside).
__device__ __forceinline__ uint32_t after_push(int sp, const double4& p_old, double3& xn, double4& vn,
                                               const Params& P, RunRec* rec, bool absorb_on, double gx,
                                               double gy, double gz)
{
	uint32_t reason = 0;
	bool hit = false;
	if (absorb_on && sp != SP_DUST) {
		const double ddx = dsub(xn.x, p_old.x), ddy = dsub(xn.y, p_old.y), ddz = dsub(xn.z, p_old.z);
		hit = P.shape ? cross_spheroid(P, xn.x, xn.y, xn.z, ddx, ddy, ddz, gx, gy, gz)
		              : cross_grain(xn.x, xn.y, xn.z, ddx, ddy, ddz, gx, gy, gz, P.a);
	}
	if (hit) {
		tally_absorbed(rec, sp, vn, P);
		reason = 1;
	} else if (P.bounce > 0.0) {
		count_wall(rec, bounce_wall(p_old, xn, vn, P));
	} else if (outside_domain(xn.x, xn.y, xn.z, P)) {
		reason = 2;
	}
	return reason;
}

}  // namespace pot
