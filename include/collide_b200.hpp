// collide_b200.hpp — header-only C++ mirror of the reference's public classes
// (uwsbel/collision-detection: src/aabb/AABBGenerator.cuh,
// src/broadphase/Broadphase.cuh, src/narrowphase/Narrowphase.cuh) over the C
// ABI in collide_b200.h, for GPU builds (custom_vector = thrust::device_vector,
// as with SIM_ENABLE_GPU_MODE, collision_detection.h:60-63).
//
// Reference call sites compile unchanged against this header (include it
// instead of Broadphase.cuh / Narrowphase.cuh / AABBGenerator.cuh and link
// libcollide_b200.so). Behaviour kept from the reference:
//  - GenerateAABB resizes aabb_data to 2N (AABBGenerator.cu:150);
//  - detectPossibleCollisions shifts aabb_data in place (Broadphase.cu:382-386),
//    resizes potentialCollisions to the unique pair count and returns 0;
//  - DoNarrowphase resizes the five outputs to the contact count and permutes
//    potentialCollisions (Narrowphase.cu:584-593);
//  - setParallelConfiguration / setBodyPerBin are stored and reported; on the
//    GPU they change nothing (the reference used them for host-side Thrust
//    dispatch and for dead code, Broadphase.cu:458-468).
// Difference: errors the reference never reports (non-finite or inverted
// boxes, out-of-range body ids, CUDA failures) throw collide_b200::Error.
#pragma once

#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include <iostream>
#include <stdexcept>
#include <string>

#include "collide_b200.h"

namespace collide_b200 {

enum shape_type { SPHERE, ELLIPSOID, BOX, CYLINDER, RECT, CONE, TRIANGLEMESH };
typedef float real;
typedef float3 real3;
typedef float4 real4;
typedef unsigned int uint;
template <class T>
using custom_vector = thrust::device_vector<T>;

class Error : public std::runtime_error {
   public:
	Error(cc_status s, const std::string &what) : std::runtime_error(what), status(s) {}
	cc_status status;
};

// One library context per device and host thread.
inline cc_ctx *context() {
	thread_local cc_ctx *ctx = nullptr;
	thread_local int dev = -1;
	int d = 0;
	cudaGetDevice(&d);
	if (!ctx || dev != d) {
		if (cc_ctx_create(&ctx, d) != CC_OK) throw Error(CC_ERR_CUDA, "cc_ctx_create failed");
		dev = d;
	}
	return ctx;
}

inline void check(cc_status s, const char *what) {
	if (s != CC_OK) throw Error(s, std::string(what) + ": " + cc_status_string(s) + " — " + cc_last_error(context()));
}

template <class T>
inline T *raw(custom_vector<T> &v) { return thrust::raw_pointer_cast(v.data()); }
template <class T>
inline const T *raw(const custom_vector<T> &v) { return thrust::raw_pointer_cast(v.data()); }
template <class T, class U>
inline const U *as(const custom_vector<T> &v) { return reinterpret_cast<const U *>(raw(v)); }
template <class T, class U>
inline U *as(custom_vector<T> &v) { return reinterpret_cast<U *>(raw(v)); }

class AABBGenerator {
   public:
	AABBGenerator() {}
	void GenerateAABB(const custom_vector<shape_type> &obj_data_T, const custom_vector<real3> &obj_data_A,
	                  const custom_vector<real3> &obj_data_B, const custom_vector<real3> &obj_data_C,
	                  const custom_vector<real4> &obj_data_R, const custom_vector<uint> &obj_data_ID,
	                  const custom_vector<real3> &body_pos, const custom_vector<real4> &body_rot,
	                  custom_vector<real3> &aabb_data) {
		numAABB = (uint)obj_data_T.size();
		aabb_data.resize(numAABB * 2);
		check(cc_generate_aabb(context(), numAABB, as<shape_type, int32_t>(obj_data_T), as<real3, float>(obj_data_A),
		                       as<real3, float>(obj_data_B), as<real3, float>(obj_data_C),
		                       as<real4, float>(obj_data_R), as<uint, uint32_t>(obj_data_ID), body_pos.size(),
		                       as<real3, float>(body_pos), as<real4, float>(body_rot), as<real3, float>(aabb_data),
		                       nullptr),
		      "GenerateAABB");
	}

   private:
	uint numAABB = 0;
};

class Broadphase {
   public:
	Broadphase() { setParallelConfiguration(1, 0, 1, 0, 0, 0, 0, 0, 1, 0); }

	int detectPossibleCollisions(custom_vector<real3> &aabb_data, custom_vector<long long> &potentialCollisions) {
		const uint64_t n = aabb_data.size() / 2;
		potentialCollisions.clear();
		uint64_t P = 0;
		cc_status s = cc_broadphase(context(), n, as<real3, float>(aabb_data), grid_size.x, grid_size.y, grid_size.z,
		                            nullptr, 0, &P, nullptr);
		if (s == CC_ERR_CAPACITY || (s == CC_OK && P > 0)) {
			potentialCollisions.resize(P);
			s = cc_broadphase_fetch(context(), reinterpret_cast<int64_t *>(raw(potentialCollisions)), P, nullptr);
		}
		check(s, "detectPossibleCollisions");
		number_of_contacts_possible = (uint)P;
		return 0;
	}
	int setBinsPerAxis(int3 binsPerAxis) {
		grid_size = binsPerAxis;
		return 0;
	}
	int3 getBinsPerAxis() { return grid_size; }
	int setBodyPerBin(int max, int min) {
		max_body_per_bin = max;
		min_body_per_bin = min;
		return 0;
	}
	int getMaxBodyPerBin() { return max_body_per_bin; }
	int getMinBodyPerBin() { return min_body_per_bin; }
	uint getNumPossibleContacts() { return number_of_contacts_possible; }
	void setParallelConfiguration(bool a, bool b, bool c, bool d, bool e, bool f, bool g, bool h, bool i, bool j) {
		const bool v[10] = {a, b, c, d, e, f, g, h, i, j};
		for (int k = 0; k < 10; k++) par[k] = v[k];
	}
	void getParallelConfiguration() {
		for (int k = 0; k < 10; k++) std::cout << par[k] << " ";
	}

   private:
	int3 grid_size = make_int3(16, 16, 16);  // Broadphase.cu:37
	int min_body_per_bin = 25, max_body_per_bin = 50;
	uint number_of_contacts_possible = 0;
	bool par[10];
};

class Narrowphase {
   public:
	Narrowphase() {}
	void DoNarrowphase(const custom_vector<shape_type> &obj_data_T, const custom_vector<real3> &obj_data_A,
	                   const custom_vector<real3> &obj_data_B, const custom_vector<real3> &obj_data_C,
	                   const custom_vector<real4> &obj_data_R, const custom_vector<uint> &obj_data_ID,
	                   const custom_vector<bool> &obj_active, const custom_vector<real3> &body_pos,
	                   const custom_vector<real4> &body_rot, custom_vector<long long> &potentialCollisions,
	                   custom_vector<real3> &norm_data, custom_vector<real3> &cpta_data,
	                   custom_vector<real3> &cptb_data, custom_vector<real> &dpth_data,
	                   custom_vector<int2> &bids_data, uint &number_of_contacts) {
		const uint64_t P = potentialCollisions.size();
		norm_data.resize(P);
		cpta_data.resize(P);
		cptb_data.resize(P);
		dpth_data.resize(P);
		bids_data.resize(P);
		uint64_t nc = 0;
		check(cc_narrowphase(context(), obj_data_T.size(), as<shape_type, int32_t>(obj_data_T),
		                     as<real3, float>(obj_data_A), as<real3, float>(obj_data_B), as<real3, float>(obj_data_C),
		                     as<real4, float>(obj_data_R), as<uint, uint32_t>(obj_data_ID), body_pos.size(),
		                     as<bool, uint8_t>(obj_active), as<real3, float>(body_pos), as<real4, float>(body_rot),
		                     collision_envelope, reinterpret_cast<int64_t *>(raw(potentialCollisions)), P,
		                     as<real3, float>(norm_data), as<real3, float>(cpta_data), as<real3, float>(cptb_data),
		                     raw(dpth_data), as<int2, int32_t>(bids_data), &nc, nullptr),
		      "DoNarrowphase");
		number_of_contacts = (uint)nc;
		norm_data.resize(nc);
		cpta_data.resize(nc);
		cptb_data.resize(nc);
		dpth_data.resize(nc);
		bids_data.resize(nc);
	}
	void SetCollisionEnvelope(const real &envelope) { collision_envelope = envelope; }
	real GetCollisionEnvelope() { return collision_envelope; }

   private:
	real collision_envelope = 0;  // Narrowphase.cu:505-509
};

}  // namespace collide_b200
