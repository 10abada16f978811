// The reference's test programs (test/test1.cu, test/binTest_Broadphase.cu,
// test/nSquared_Broadphase.cu, test/timing_Broadphase.cu), written against
// include/collide_b200.hpp: the same class calls a Chrono-side caller makes,
// now on the B200 library. Usage: reference_tests [test1|bintest|nsquared|
// timing|pipeline|all]. Prints TEST PASSED / TEST FAILED like the originals;
// the exit code is the number of failures.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <vector>

#include "collide_b200.hpp"

using namespace collide_b200;

static double rnd(double lo, double hi) { return lo + (rand() / (double)RAND_MAX) * (hi - lo); }

struct Sphere {
	double r;
	real3 pos;
};

static void sphere_aabbs(const std::vector<Sphere> &s, custom_vector<real3> &aabb) {
	std::vector<real3> h(2 * s.size());
	for (size_t i = 0; i < s.size(); i++) {
		real3 lo = s[i].pos, hi = s[i].pos;
		lo.x -= s[i].r; lo.y -= s[i].r; lo.z -= s[i].r;
		hi.x += s[i].r; hi.y += s[i].r; hi.z += s[i].r;
		h[i] = lo;
		h[i + s.size()] = hi;
	}
	aabb = h;
}

// test/test1.cu: n identical unit boxes in one bin -> n(n-1)/2 pairs
static int test1(int n) {
	std::vector<real3> h;
	for (int i = 0; i < n; i++) h.push_back(make_float3(0, 0, 0));
	for (int i = 0; i < n; i++) h.push_back(make_float3(1, 1, 1));
	custom_vector<real3> aabb = h;
	custom_vector<long long> pc;
	Broadphase bp;
	bp.setBinsPerAxis(make_int3(1, 1, 1));
	bp.detectPossibleCollisions(aabb, pc);
	bool ok = pc.size() == (size_t)n * (n - 1) / 2 && bp.getNumPossibleContacts() == pc.size();
	printf("test1 n=%d pairs=%zu %s\n", n, pc.size(), ok ? "TEST PASSED" : "TEST FAILED");
	return ok ? 0 : 1;
}

// test/binTest_Broadphase.cu: every lattice sphere listed twice -> m^3 pairs
static int bintest(int m, int bpa) {
	std::vector<Sphere> s;
	for (int k = 0; k < m; k++)
		for (int j = 0; j < m; j++)
			for (int i = 0; i < m; i++) {
				Sphere sp = {0.25, make_float3(i, j, k)};
				s.push_back(sp);
				s.push_back(sp);
			}
	custom_vector<real3> aabb;
	sphere_aabbs(s, aabb);
	custom_vector<long long> pc;
	Broadphase bp;
	bp.setBinsPerAxis(make_int3(bpa, bpa, bpa));
	bp.detectPossibleCollisions(aabb, pc);
	bool ok = bp.getNumPossibleContacts() == (uint)(m * m * m);
	printf("binTest m=%d bpa=%d pairs=%u %s\n", m, bpa, bp.getNumPossibleContacts(), ok ? "TEST PASSED" : "TEST FAILED");
	return ok ? 0 : 1;
}

// test/nSquared_Broadphase.cu: every true overlap (strict, double) is found
static int nsquared(int n) {
	srand(1);
	std::vector<Sphere> s(n);
	for (int i = 0; i < n; i++) {
		s[i].pos = make_float3(rnd(-30, 30), rnd(-30, 30), rnd(-30, 30));
		s[i].r = rnd(.1, 1);
	}
	custom_vector<real3> aabb;
	sphere_aabbs(s, aabb);
	custom_vector<long long> pc;
	Broadphase bp;
	bp.setBinsPerAxis(make_int3(30, 30, 30));
	bp.detectPossibleCollisions(aabb, pc);
	std::vector<long long> h(pc.size());
	thrust::copy(pc.begin(), pc.end(), h.begin());
	size_t missed = 0, truth = 0;
	for (int i = 0; i < n; i++)
		for (int j = i + 1; j < n; j++) {
			double d = pow(s[i].pos.x - s[j].pos.x, 2.0) + pow(s[i].pos.y - s[j].pos.y, 2.0) +
			           pow(s[i].pos.z - s[j].pos.z, 2.0);
			if (d < pow(s[i].r + s[j].r, 2.0)) {
				truth++;
				long long key = ((long long)i << 32) | j;
				if (!std::binary_search(h.begin(), h.end(), key)) missed++;
			}
		}
	bool ok = missed == 0 && truth > 0;
	printf("nSquared n=%d pairs=%zu true=%zu missed=%zu %s\n", n, h.size(), truth, missed,
	       ok ? "TEST PASSED" : "TEST FAILED");
	return ok ? 0 : 1;
}

// test/timing_Broadphase.cu: 300k spheres, 50^3 bins, average of 10 calls
static int timing() {
	srand(2);
	const int n = 300000;
	std::vector<Sphere> s(n);
	for (int i = 0; i < n; i++) {
		s[i].pos = make_float3(rnd(-30, 30), rnd(-30, 30), rnd(-30, 30));
		s[i].r = rnd(.1, 1);
	}
	custom_vector<real3> aabb0, aabb;
	sphere_aabbs(s, aabb0);
	custom_vector<long long> pc;
	double total = 0;
	uint P = 0;
	for (int rep = 0; rep < 11; rep++) {
		aabb = aabb0;  // the call shifts its input in place
		Broadphase bp;
		bp.setBinsPerAxis(make_int3(50, 50, 50));
		cudaDeviceSynchronize();
		auto t0 = std::chrono::steady_clock::now();
		bp.detectPossibleCollisions(aabb, pc);
		cudaDeviceSynchronize();
		auto t1 = std::chrono::steady_clock::now();
		if (rep) total += std::chrono::duration<double>(t1 - t0).count();
		P = bp.getNumPossibleContacts();
	}
	printf("timing n=%d avg_time=%.6f s pairs=%u\n", n, total / 10, P);
	return 0;
}

// GenerateAABB -> detectPossibleCollisions -> DoNarrowphase, the Chrono sequence
static int pipeline() {
	srand(3);
	const int n = 20000;
	std::vector<shape_type> T(n);
	std::vector<real3> A(n, make_float3(0, 0, 0)), B(n), C(n, make_float3(0, 0, 0)), pos(n);
	std::vector<real4> R(n, make_float4(1, 0, 0, 0)), rot(n);
	std::vector<uint> ID(n);
	std::vector<char> act(n, 1);
	for (int i = 0; i < n; i++) {
		T[i] = (shape_type)(i % 4);
		double r = rnd(0.01, 0.04);
		B[i] = T[i] == SPHERE ? make_float3(r, 0, 0) : make_float3(rnd(0.01, 0.04), rnd(0.01, 0.04), r);
		if (T[i] == CYLINDER) B[i].z = B[i].x;
		pos[i] = make_float3(rnd(0, 2), rnd(0, 2), rnd(0, 0.2));
		double q[4] = {rnd(-1, 1), rnd(-1, 1), rnd(-1, 1), rnd(-1, 1)};
		double l = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
		rot[i] = make_float4(q[0] / l, q[1] / l, q[2] / l, q[3] / l);
		ID[i] = i;
	}
	custom_vector<shape_type> dT = T;
	custom_vector<real3> dA = A, dB = B, dC = C, dpos = pos, aabb;
	custom_vector<real4> dR = R, drot = rot;
	custom_vector<uint> dID = ID;
	custom_vector<bool> dact(n, true);
	AABBGenerator gen;
	gen.GenerateAABB(dT, dA, dB, dC, dR, dID, dpos, drot, aabb);
	Broadphase bp;
	custom_vector<long long> pc;
	bp.detectPossibleCollisions(aabb, pc);
	Narrowphase np;
	custom_vector<real3> norm, cpta, cptb;
	custom_vector<real> depth;
	custom_vector<int2> bids;
	uint nc = 0;
	np.DoNarrowphase(dT, dA, dB, dC, dR, dID, dact, dpos, drot, pc, norm, cpta, cptb, depth, bids, nc);
	std::vector<real3> hn(norm.size());
	thrust::copy(norm.begin(), norm.end(), hn.begin());
	bool ok = nc > 0 && nc <= bp.getNumPossibleContacts() && norm.size() == nc && depth.size() == nc;
	for (uint i = 0; i < nc && ok; i++) {
		double l = sqrt(hn[i].x * hn[i].x + hn[i].y * hn[i].y + hn[i].z * hn[i].z);
		ok = fabs(l - 1.0) < 1e-5;
	}
	printf("pipeline n=%d pairs=%u contacts=%u %s\n", n, bp.getNumPossibleContacts(), nc,
	       ok ? "TEST PASSED" : "TEST FAILED");
	return ok ? 0 : 1;
}

int main(int argc, char **argv) {
	const char *which = argc > 1 ? argv[1] : "all";
	int fails = 0;
	bool all = !strcmp(which, "all");
	if (all || !strcmp(which, "test1")) fails += test1(10) + test1(300);
	if (all || !strcmp(which, "bintest")) fails += bintest(10, 10) + bintest(20, 7);
	if (all || !strcmp(which, "nsquared")) fails += nsquared(20000);
	if (all || !strcmp(which, "pipeline")) fails += pipeline();
	if (!strcmp(which, "timing")) fails += timing();
	return fails;
}
