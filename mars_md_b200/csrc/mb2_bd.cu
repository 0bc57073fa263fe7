// Brownian-dynamics integrator with the fused position-dependent force.
//
// Replaces BDIntegrate<float> (src/PatchOperation/Integrator/BD.h:44-92) with
// compute_position_dependent_force (src/Interactions/Nonbonded/Pmf.h:68-124)
// and the trilinear grid sampling of src/Types/BaseGridDevice.h:218-365.
//
// Per particle: skip FLAG_RB_ATTACHED; F += q E + sum over the type's PMF
// terms of -scale * grad U (energy scale * U into .w) + per-axis force grids;
// Philox4x32-10 with key = base_seed and counter (base_ctr + slot, 0x5324120,
// step, 0); Box-Muller; x += (D/kT) F dt + sqrt(2 D dt) xi per axis; wrap.
// The Philox integers are bit-identical to the reference; logf/sinf/cosf are
// CUDA's (not fast-math), within a few ulp of the host libm the reference's
// CPU build uses.
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

// map_grid_index (BaseGridDevice.h:218-232).
__device__ __forceinline__ bool map_index(int& j, long long n, int bc) {
	const int ni = static_cast<int>(n);
	if (j >= 0 && j < ni) return true;
	if (bc == 2) {
		j = ((j % ni) + ni) % ni;
		return true;
	}
	if (bc == 1) {
		j = j < 0 ? 0 : ni - 1;
		return true;
	}
	return false;
}

// fetch_grid_value (BaseGridDevice.h:479-500) for the 2 x 2 x 2 taps of a
// trilinear sample at (i0, j0, k0): each axis' two indices are mapped once,
// and all eight loads are issued before any is used (a tap outside a
// Dirichlet grid reads element 0 and is replaced by 0), so the taps' memory
// latencies overlap instead of following one another.
__device__ __forceinline__ void fetch8(const GridView& g, int i0, int j0, int k0, int bc,
									   float v[8]) {
	int ix[2] = {i0, i0 + 1}, iy[2] = {j0, j0 + 1}, iz[2] = {k0, k0 + 1};
	bool ox[2], oy[2], oz[2];
#pragma unroll
	for (int t = 0; t < 2; ++t) {
		ox[t] = map_index(ix[t], g.dims[0], bc);
		oy[t] = map_index(iy[t], g.dims[1], bc);
		oz[t] = map_index(iz[t], g.dims[2], bc);
	}
	const size_t ny = static_cast<size_t>(g.dims[1]), nz = static_cast<size_t>(g.dims[2]);
	bool ok[8];
#pragma unroll
	for (int t = 0; t < 8; ++t) {
		const int a = t >> 2, b = (t >> 1) & 1, c = t & 1;  // tap (x, y, z) = (a, b, c)
		ok[t] = ox[a] && oy[b] && oz[c];
		const size_t idx = ok[t] ? static_cast<size_t>(iz[c]) + static_cast<size_t>(iy[b]) * nz +
									   static_cast<size_t>(ix[a]) * ny * nz
								 : 0;
		v[t] = __ldg(g.data + idx);
	}
#pragma unroll
	for (int t = 0; t < 8; ++t)
		if (!ok[t]) v[t] = 0.0f;
}

// Trilinear value and analytic gradient (interpolate_grid_point and
// compute_gradient, BaseGridDevice.h:256-365), same operation order.
__device__ __forceinline__ void grid_sample(const GridView& g, float px, float py, float pz, int bc,
											float& value, float3& grad) {
	const float dx = __fsub_rn(px, g.origin[0]), dy = __fsub_rn(py, g.origin[1]),
				dz = __fsub_rn(pz, g.origin[2]);
	const float* m = g.basis_inv;  // column-major
	float gp[3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
		gp[r] = __fadd_rn(__fadd_rn(__fmul_rn(dx, m[r]), __fmul_rn(dy, m[3 + r])),
						  __fmul_rn(dz, m[6 + r]));
	const int i0 = static_cast<int>(floorf(gp[0]));
	const int j0 = static_cast<int>(floorf(gp[1]));
	const int k0 = static_cast<int>(floorf(gp[2]));
	const float fx = __fsub_rn(gp[0], static_cast<float>(i0));
	const float fy = __fsub_rn(gp[1], static_cast<float>(j0));
	const float fz = __fsub_rn(gp[2], static_cast<float>(k0));
	float v[8];
	fetch8(g, i0, j0, k0, bc, v);
	const float v000 = v[0], v001 = v[1], v010 = v[2], v011 = v[3];
	const float v100 = v[4], v101 = v[5], v110 = v[6], v111 = v[7];
	const float ox = __fsub_rn(1.0f, fx), oy = __fsub_rn(1.0f, fy), oz = __fsub_rn(1.0f, fz);
	auto lerp = [](float a, float wa, float b, float wb) {
		return __fadd_rn(__fmul_rn(a, wa), __fmul_rn(b, wb));
	};
	const float v00 = lerp(v000, ox, v100, fx), v01 = lerp(v001, ox, v101, fx);
	const float v10 = lerp(v010, ox, v110, fx), v11 = lerp(v011, ox, v111, fx);
	const float v0 = lerp(v00, oy, v10, fy), v1 = lerp(v01, oy, v11, fy);
	value = lerp(v0, oz, v1, fz);
	auto term = [](float w1, float w2, float d) { return __fmul_rn(__fmul_rn(w1, w2), d); };
	const float gx = __fadd_rn(__fadd_rn(__fadd_rn(term(oy, oz, __fsub_rn(v100, v000)),
												   term(fy, oz, __fsub_rn(v110, v010))),
										 term(oy, fz, __fsub_rn(v101, v001))),
							   term(fy, fz, __fsub_rn(v111, v011)));
	const float gy = __fadd_rn(__fadd_rn(__fadd_rn(term(ox, oz, __fsub_rn(v010, v000)),
												   term(fx, oz, __fsub_rn(v110, v100))),
										 term(ox, fz, __fsub_rn(v011, v001))),
							   term(fx, fz, __fsub_rn(v111, v101)));
	const float gz = __fadd_rn(__fadd_rn(__fadd_rn(term(ox, oy, __fsub_rn(v001, v000)),
												   term(fx, oy, __fsub_rn(v101, v100))),
										 term(ox, fy, __fsub_rn(v011, v010))),
							   term(fx, fy, __fsub_rn(v111, v110)));
	// transpose(basis_inv).transform(g): row r of basis_inv dotted with g
	grad.x = __fadd_rn(__fadd_rn(__fmul_rn(gx, m[0]), __fmul_rn(gy, m[1])), __fmul_rn(gz, m[2]));
	grad.y = __fadd_rn(__fadd_rn(__fmul_rn(gx, m[3]), __fmul_rn(gy, m[4])), __fmul_rn(gz, m[5]));
	grad.z = __fadd_rn(__fadd_rn(__fmul_rn(gx, m[6]), __fmul_rn(gy, m[7])), __fmul_rn(gz, m[8]));
}

// compute_position_dependent_force (Pmf.h:68-124). kGrids false: the caller
// knows that no grid is loaded (ty.num_grids == 0), and the grid code is not
// compiled in.
template <bool kGrids = true>
__device__ __forceinline__ float4 position_force(const TypeTable& ty, int type, float px, float py,
												 float pz, const float* efield) {
	const float q = ty.charge[type];
	float4 f = make_float4(__fmul_rn(q, efield[0]), __fmul_rn(q, efield[1]),
						   __fmul_rn(q, efield[2]), 0.0f);
	if (!kGrids || ty.num_grids == 0) return f;
	const int begin = ty.pmf_offset[type];
	const int end = begin + ty.pmf_count[type];
	for (int k = begin; k < end; ++k) {
		const GridTermDev term = ty.terms[k];
		if (term.grid_id < 0) continue;
		const GridView& g = ty.grids[term.grid_id];
		if (g.data == nullptr) continue;
		const int bc = term.boundary_condition >= 0 ? term.boundary_condition : g.boundary_condition;
		float value;
		float3 grad;
		grid_sample(g, px, py, pz, bc, value, grad);
		const float s = -term.scale;
		f.x = __fadd_rn(f.x, __fmul_rn(grad.x, s));
		f.y = __fadd_rn(f.y, __fmul_rn(grad.y, s));
		f.z = __fadd_rn(f.z, __fmul_rn(grad.z, s));
		f.w = __fadd_rn(f.w, __fmul_rn(term.scale, value));
	}
	const int4 fg = ty.force_grid_id[type];
	const float4 fs = ty.force_grid_scale[type];
	const int ids[3] = {fg.x, fg.y, fg.z};
	const float sc[3] = {fs.x, fs.y, fs.z};
	float* comp[3] = {&f.x, &f.y, &f.z};
#pragma unroll
	for (int a = 0; a < 3; ++a) {
		if (ids[a] < 0) continue;
		const GridView& g = ty.grids[ids[a]];
		if (g.data == nullptr) continue;
		float value;
		float3 grad;
		grid_sample(g, px, py, pz, g.boundary_condition, value, grad);
		*comp[a] = __fadd_rn(*comp[a], __fmul_rn(sc[a], value));
	}
	return f;
}

// Box-Muller of one Philox draw (BD.h:66-78; BAOAB.h:98-110 with its own stream).
__device__ __forceinline__ float3 bd_noise(uint64_t seed, uint32_t ctr, uint32_t step,
										   uint32_t stream = kBdStream) {
	const uint4 u = philox4x32_10(seed, ctr, stream, step, 0u);
	const float ux = u01(u.x), uy = u01(u.y), uz = u01(u.z), uw = u01(u.w);
	const float r1 = __fsqrt_rn(__fmul_rn(-2.0f, logf(ux)));
	const float t1 = __fmul_rn(6.2831854820251465f, uy);  // 2.0f * 3.1415926535f
	const float r2 = __fsqrt_rn(__fmul_rn(-2.0f, logf(uz)));
	const float t2 = __fmul_rn(6.2831854820251465f, uw);
	float s1, c1;
	sincosf(t1, &s1, &c1);
	return make_float3(__fmul_rn(r1, c1), __fmul_rn(r1, s1), __fmul_rn(r2, cosf(t2)));
}

// x + ((D / kT) F dt + sqrt(2 D dt) xi), as BD.h:80-85 groups it.
__device__ __forceinline__ float bd_axis(float x, float d, float kT, float f, float dt, float xi) {
	const float drift = __fmul_rn(__fmul_rn(__fdiv_rn(d, kT), f), dt);
	const float noise = __fmul_rn(__fsqrt_rn(__fmul_rn(__fmul_rn(2.0f, d), dt)), xi);
	return __fadd_rn(x, __fadd_rn(drift, noise));
}

__device__ __forceinline__ float4 bd_update(float4 p, float fx, float fy, float fz, const float4& dif,
											const float3& xi, const Box& box, const BdParams& bp) {
	p.x = bd_axis(p.x, dif.x, bp.kT, fx, bp.dt, xi.x);
	p.y = bd_axis(p.y, dif.y, bp.kT, fy, bp.dt, xi.y);
	p.z = bd_axis(p.z, dif.z, bp.kT, fz, bp.dt, xi.z);
	if (box.periodic[0]) p.x = wrap_scalar(p.x, box.origin[0], box.size[0], box.inv[0]);
	if (box.periodic[1]) p.y = wrap_scalar(p.y, box.origin[1], box.size[1], box.inv[1]);
	if (box.periodic[2]) p.z = wrap_scalar(p.z, box.origin[2], box.size[2], box.inv[2]);
	return p;
}

__global__ void __launch_bounds__(256) bd_kernel(float4* __restrict__ pos, float4* __restrict__ fe,
												 const int* __restrict__ type_ids,
												 const uint32_t* __restrict__ flags, uint32_t n,
												 TypeTable ty, Box box, BdParams bp) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (flags && (flags[i] & kFlagRbAttached)) return;
	float4 p = pos[i];
	float4 f = fe[i];
	const int type = type_ids[i];
	const float4 pmf = position_force(ty, type, p.x, p.y, p.z, bp.efield);
	f.x = __fadd_rn(f.x, pmf.x);
	f.y = __fadd_rn(f.y, pmf.y);
	f.z = __fadd_rn(f.z, pmf.z);
	if (pmf.w != 0.0f) fe[i].w = __fadd_rn(f.w, pmf.w);
	const float3 xi = bd_noise(bp.base_seed, bp.base_ctr + i, bp.step);
	pos[i] = bd_update(p, f.x, f.y, f.z, ty.diffusion[type], xi, box, bp);
}

__device__ __forceinline__ uint64_t mix_seed(uint64_t seed, uint64_t patch, uint64_t step) {
	// Patch::integrate_motion seed mixing (Patch.cpp:252-254).
	return (seed * 0x9E3779B97F4A7C15ULL) ^ (patch << 32) ^ (step * 0xBF58476D1CE4E5B9ULL);
}

// Fused-step variant: the pair force is gathered from the Z-ordered
// accumulator through the inverse permutation (random reads, coalesced
// writes), added to what the bonded kernels left in ForceEnergy when any ran
// (read_fe), and the result stored to ForceEnergy as the reference leaves it
// after integrate_motion; then the grid force, noise and update as bd_kernel.
// step_ptr (graph replay): the step number comes from device memory and the
// Philox key is mixed here from (seed, patch_id, step), as the host does for
// bp.base_seed otherwise. kGrids false (no grid loaded): without the grid
// code the kernel takes fewer registers and more warps fit on an SM.
template <bool kGrids>
__global__ void __launch_bounds__(256) bd_gather_kernel(
	float4* __restrict__ pos, float4* __restrict__ fe, const float4* __restrict__ fs,
	const uint32_t* __restrict__ inv, const int* __restrict__ type_ids,
	const uint32_t* __restrict__ flags, uint32_t n, TypeTable ty, Box box, BdParams bp,
	int read_fe, const unsigned long long* __restrict__ step_ptr, uint64_t seed,
	uint64_t patch_id) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (step_ptr) {
		const uint64_t step = *step_ptr;
		bp.step = static_cast<uint32_t>(step);
		bp.base_seed = mix_seed(seed, patch_id, step);
	}
	float4 f = fs[inv[i]];
	if (read_fe) {
		const float4 ext = fe[i];
		f.x = __fadd_rn(ext.x, f.x);
		f.y = __fadd_rn(ext.y, f.y);
		f.z = __fadd_rn(ext.z, f.z);
		f.w = __fadd_rn(ext.w, f.w);
	}
	if (flags && (flags[i] & kFlagRbAttached)) {
		fe[i] = f;
		return;
	}
	const float4 p = pos[i];
	const int type = type_ids[i];
	const float4 pmf = position_force<kGrids>(ty, type, p.x, p.y, p.z, bp.efield);
	const float3 xi = bd_noise(bp.base_seed, bp.base_ctr + i, bp.step);
	if (pmf.w != 0.0f) f.w = __fadd_rn(f.w, pmf.w);
	fe[i] = f;
	pos[i] = bd_update(p, __fadd_rn(f.x, pmf.x), __fadd_rn(f.y, pmf.y), __fadd_rn(f.z, pmf.z),
					   ty.diffusion[type], xi, box, bp);
}

// FORCE_CONVERSION_FACTOR, SQRT_CAL_TO_JOULE (src/Constants.h:30,34) and the
// BAOAB noise stream (BAOAB.h:30).
constexpr float kForceConversion = 4.18679994e4f;
constexpr float kSqrtCalToJoule = 2.046167337f;
constexpr uint32_t kBaoabStream = 0x1356914u;

// mom += (0.5 dt F) * FORCE_CONVERSION_FACTOR, as Vector3 arithmetic rounds it.
__device__ __forceinline__ float half_kick(float m, float f, float h) {
	return __fadd_rn(m, __fmul_rn(__fmul_rn(h, f), kForceConversion));
}

// Patch::integrate_motion's Langevin branch (Patch.cpp:290-335) for one
// particle: PMF pass (Pmf.h:126-152), closing kick if pending (BAOAB.h:167-186),
// then BAOABIntegrate (BAOAB.h:47-128). Vector3 / s is a multiply by 1 / s.
// kGather (the fused step): the pair force comes from the Z-ordered
// accumulator through the inverse permutation, plus what the bonded kernels
// left in ForceEnergy when any ran (read_fe), and ForceEnergy receives the
// sum as the reference leaves it.
template <bool kGather>
__global__ void __launch_bounds__(256) baoab_kernel(
	float4* __restrict__ pos, float4* __restrict__ mom, float4* __restrict__ fe,
	const float4* __restrict__ fs, const uint32_t* __restrict__ inv, int read_fe,
	const int* __restrict__ type_ids, const uint32_t* __restrict__ flags, uint32_t n,
	TypeTable ty, Box box, float dt, float kT, uint32_t step, uint64_t seed, uint32_t base_ctr,
	float3 efield, int pending) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	float4 p = pos[i];
	float4 f;
	if (kGather) {
		f = fs[inv[i]];
		if (read_fe) {
			const float4 ext = fe[i];
			f.x = __fadd_rn(ext.x, f.x);
			f.y = __fadd_rn(ext.y, f.y);
			f.z = __fadd_rn(ext.z, f.z);
			f.w = __fadd_rn(ext.w, f.w);
		}
	} else {
		f = fe[i];
	}
	const int type = type_ids[i];
	if (ty.num_grids > 0) {
		const float e[3] = {efield.x, efield.y, efield.z};
		const float4 pmf = position_force(ty, type, p.x, p.y, p.z, e);
		f.x = __fadd_rn(f.x, pmf.x);
		f.y = __fadd_rn(f.y, pmf.y);
		f.z = __fadd_rn(f.z, pmf.z);
		f.w = __fadd_rn(f.w, pmf.w);
		if (!kGather) fe[i] = f;
	}
	if (kGather) fe[i] = f;
	if (flags && (flags[i] & kFlagRbAttached)) return;
	float4 m = mom[i];
	const float h = __fmul_rn(0.5f, dt);
	if (pending) {
		m.x = half_kick(m.x, f.x, h);
		m.y = half_kick(m.y, f.y, h);
		m.z = half_kick(m.z, f.z, h);
	}
	m.x = half_kick(m.x, f.x, h);  // B
	m.y = half_kick(m.y, f.y, h);
	m.z = half_kick(m.z, f.z, h);
	const float ms = ty.mass[type];
	const float inv_m = __fdiv_rn(1.0f, ms);
	auto drift = [&](float x, float mv) {
		return __fadd_rn(x, __fmul_rn(__fmul_rn(__fmul_rn(h, mv), inv_m), 10000.0f));
	};
	p.x = drift(p.x, m.x);  // A
	p.y = drift(p.y, m.y);
	p.z = drift(p.z, m.z);
	const float4 g = ty.damping[type];
	const float3 xi = bd_noise(seed, base_ctr + i, step, kBaoabStream);
	auto ou = [&](float mv, float gamma, float r) {  // O
		const float c = expf(__fmul_rn(-gamma, dt));
		const float ns = __fmul_rn(
			__fsqrt_rn(__fmul_rn(__fmul_rn(kT, ms), __fsub_rn(1.0f, __fmul_rn(c, c)))),
			kSqrtCalToJoule);
		return __fadd_rn(__fmul_rn(c, mv), __fmul_rn(ns, r));
	};
	m.x = ou(m.x, g.x, xi.x);
	m.y = ou(m.y, g.y, xi.y);
	m.z = ou(m.z, g.z, xi.z);
	p.x = drift(p.x, m.x);  // A
	p.y = drift(p.y, m.y);
	p.z = drift(p.z, m.z);
	if (box.periodic[0]) p.x = wrap_scalar(p.x, box.origin[0], box.size[0], box.inv[0]);
	if (box.periodic[1]) p.y = wrap_scalar(p.y, box.origin[1], box.size[1], box.inv[1]);
	if (box.periodic[2]) p.z = wrap_scalar(p.z, box.origin[2], box.size[2], box.inv[2]);
	pos[i] = p;
	mom[i] = m;
}

__global__ void __launch_bounds__(256) baoab_last_kernel(float4* __restrict__ mom,
														 const float4* __restrict__ fe,
														 const uint32_t* __restrict__ flags,
														 uint32_t n, float dt) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (flags && (flags[i] & kFlagRbAttached)) return;
	const float4 f = fe[i];
	float4 m = mom[i];
	const float h = __fmul_rn(0.5f, dt);
	m.x = half_kick(m.x, f.x, h);
	m.y = half_kick(m.y, f.y, h);
	m.z = half_kick(m.z, f.z, h);
	mom[i] = m;
}

// Batched replicas: particle i of system s = sys_of[i] integrates as a plain
// step of system s with seed (seed + s) would (counter = index in the
// system, its own box); the step number comes from device memory so that a
// captured graph can be replayed step after step. kGrids as bd_gather_kernel.
template <bool kGrids>
__global__ void __launch_bounds__(256) bd_systems_kernel(
	float4* __restrict__ pos, float4* __restrict__ fe, const float4* __restrict__ fs,
	const uint32_t* __restrict__ inv, const int* __restrict__ type_ids,
	const uint32_t* __restrict__ sys_of, const uint32_t* __restrict__ offsets,
	const Box* __restrict__ boxes, uint32_t n, TypeTable ty, float dt, float kT, uint64_t seed,
	uint64_t patch_id, const unsigned long long* __restrict__ step_ptr) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint64_t step = *step_ptr;
	const uint32_t s = sys_of[i];
	const Box& box = boxes[s];
	float4 f = fs[inv[i]];
	const float4 p = pos[i];
	const int type = type_ids[i];
	const BdParams bp{dt, kT, static_cast<uint32_t>(step), mix_seed(seed + s, patch_id, step), 0u,
					  {0.0f, 0.0f, 0.0f}};
	const float4 pmf = position_force<kGrids>(ty, type, p.x, p.y, p.z, bp.efield);
	const float3 xi = bd_noise(bp.base_seed, i - offsets[s], bp.step);
	if (pmf.w != 0.0f) f.w = __fadd_rn(f.w, pmf.w);
	fe[i] = f;
	pos[i] = bd_update(p, __fadd_rn(f.x, pmf.x), __fadd_rn(f.y, pmf.y), __fadd_rn(f.z, pmf.z),
					   ty.diffusion[type], xi, box, bp);
}

__global__ void step_counter_kernel(unsigned long long* ptr, unsigned long long v, int add) {
	*ptr = add ? *ptr + v : v;
}

__global__ void philox_kernel(uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2,
							  uint32_t n, uint4* out4, float4* normals4) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (out4) out4[i] = philox4x32_10(seed, ctr0 + i, ctr1, ctr2, 0u);
	if (normals4) {
		const float3 xi = bd_noise(seed, ctr0 + i, ctr2);
		normals4[i] = make_float4(xi.x, xi.y, xi.z, 0.0f);
	}
}

}  // namespace

void bd_integrate(float4* pos, float4* fe, const int* type_ids, const uint32_t* flags, uint32_t n,
				  const TypeTable& types, const Box& box, const BdParams& p, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH bd_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, fe, type_ids, flags, n, types, box, p);
}

void bd_integrate_gather(float4* pos, float4* fe, const float4* force_sorted, const uint32_t* inv,
						 const int* type_ids, const uint32_t* flags, uint32_t n,
						 const TypeTable& types, const Box& box, const BdParams& p, int read_fe,
						 cudaStream_t st, const unsigned long long* step_ptr, uint64_t seed,
						 uint64_t patch_id) {
	if (n == 0) return;
	auto kern = types.num_grids == 0 ? bd_gather_kernel<false> : bd_gather_kernel<true>;
	MB2_LAUNCH kern<<<(n + 255) / 256, 256, 0, st>>>(pos, fe, force_sorted, inv, type_ids, flags, n,
													 types, box, p, read_fe, step_ptr, seed,
													 patch_id);
}

void baoab_integrate(float4* pos, float4* mom, float4* fe, const int* type_ids,
					 const uint32_t* flags, uint32_t n, const TypeTable& types, const Box& box,
					 float dt, float kT, uint32_t step, uint64_t base_seed, uint32_t base_ctr,
					 const float* efield, int pending, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH baoab_kernel<false><<<(n + 255) / 256, 256, 0, st>>>(
		pos, mom, fe, nullptr, nullptr, 0, type_ids, flags, n, types, box, dt, kT, step, base_seed,
		base_ctr, make_float3(efield[0], efield[1], efield[2]), pending);
}

void baoab_integrate_gather(float4* pos, float4* mom, float4* fe, const float4* force_sorted,
							const uint32_t* inv, int read_fe, const int* type_ids,
							const uint32_t* flags, uint32_t n, const TypeTable& types,
							const Box& box, float dt, float kT, uint32_t step, uint64_t base_seed,
							uint32_t base_ctr, const float* efield, int pending, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH baoab_kernel<true><<<(n + 255) / 256, 256, 0, st>>>(
		pos, mom, fe, force_sorted, inv, read_fe, type_ids, flags, n, types, box, dt, kT, step,
		base_seed, base_ctr, make_float3(efield[0], efield[1], efield[2]), pending);
}

void baoab_last_update(float4* mom, const float4* fe, const uint32_t* flags, uint32_t n,
					   float dt, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH baoab_last_kernel<<<(n + 255) / 256, 256, 0, st>>>(mom, fe, flags, n, dt);
}

void bd_integrate_systems(float4* pos, float4* fe, const float4* force_sorted,
						  const uint32_t* inv, const int* type_ids, const uint32_t* sys_of,
						  const uint32_t* offsets, const Box* boxes, uint32_t n,
						  const TypeTable& types, float dt, float kT, uint64_t seed,
						  uint64_t patch_id, const unsigned long long* step_ptr, cudaStream_t st) {
	if (n == 0) return;
	auto kern = types.num_grids == 0 ? bd_systems_kernel<false> : bd_systems_kernel<true>;
	MB2_LAUNCH kern<<<(n + 255) / 256, 256, 0, st>>>(pos, fe, force_sorted, inv, type_ids, sys_of,
													 offsets, boxes, n, types, dt, kT, seed,
													 patch_id, step_ptr);
}

void step_counter_set(unsigned long long* ptr, uint64_t value, cudaStream_t st) {
	MB2_LAUNCH step_counter_kernel<<<1, 1, 0, st>>>(ptr, value, 0);
}

void step_counter_add(unsigned long long* ptr, uint64_t value, cudaStream_t st) {
	MB2_LAUNCH step_counter_kernel<<<1, 1, 0, st>>>(ptr, value, 1);
}

void philox_draws(uint64_t seed, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2, uint32_t n,
				  uint32_t* out4, float* normals4, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH philox_kernel<<<(n + 255) / 256, 256, 0, st>>>(seed, ctr0, ctr1, ctr2, n,
												   reinterpret_cast<uint4*>(out4),
												   reinterpret_cast<float4*>(normals4));
}

}  // namespace mb2
