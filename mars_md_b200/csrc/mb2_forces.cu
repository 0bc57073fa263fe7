// Tabulated pair, bond and angle forces.
//
// Pair forces replace PairNonbondedComputer's tabulated term
// (src/Interactions/Nonbonded/Pairwise.h:214-304): per pair, wrapped r_ij,
// |r_ij| by sqrt, skip |r| < 1e-6 and |r|^2 > rc^2, table lookup,
// f = r_ij / |r_ij| * F, -f on the pair's first (smaller original) index and
// +f on the second, half the energy to each. Each pair's float result is
// rounded exactly as the reference rounds it (explicit _rn intrinsics, the
// same orientation via bit 31 of the list entry); only the order in which
// the per-particle sums accumulate differs.
//
// Layout: a group of G lanes owns one row (sorted particle i) of the CSR half
// list. Lanes stride over the row, gather sorted float4 positions (type id in
// .w), accumulate -f for i in registers and scatter +f to j with one vector
// `red.global.add.v4.f32` per pair (energy rides in .w). The row's i force is
// reduced across the group with shuffles and added with one more vector red.
// Tables and the type-pair tag matrix live in shared memory.
//
// FP64: the total pair energy and virial are reduced in double on the device
// (a per-thread double, a block reduction, one double atomic per block).
#include "mb2_internal.cuh"

namespace mb2 {

namespace {

struct SmemTable {
	float start;
	float step_inv;
	int size;
	int offset;
};

__device__ __forceinline__ void block_add_f64(double a, double b, double* out) {
	__shared__ double red_a[32], red_b[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
		b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
	}
	if (lane == 0) {
		red_a[warp] = a;
		red_b[warp] = b;
	}
	__syncthreads();
	if (warp == 0) {
		const int nw = blockDim.x >> 5;
		a = lane < nw ? red_a[lane] : 0.0;
		b = lane < nw ? red_b[lane] : 0.0;
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
			b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
		}
		if (lane == 0) {
			atomicAdd(out, a);
			atomicAdd(out + 1, b);
		}
	}
}

template <int G>
__global__ void __launch_bounds__(256) pair_force_kernel(
	const float4* __restrict__ sorted_pos, const uint32_t* __restrict__ row_start,
	const uint32_t* __restrict__ nbr, uint32_t n, const uint32_t* __restrict__ term_g, int T,
	const Table* __restrict__ tables_g, int num_tables, const float* __restrict__ values_g,
	uint32_t total_values, Box box, float cutoff_sq, int get_energy, float4* force,
	double* __restrict__ ev) {
	extern __shared__ uint32_t smem[];
	uint32_t* term = smem;                                                    // T*T
	SmemTable* tabs = reinterpret_cast<SmemTable*>(smem + ((T * T + 3) & ~3)); // num_tables
	float* vals = reinterpret_cast<float*>(tabs + num_tables);               // total_values
	for (int k = threadIdx.x; k < T * T; k += blockDim.x) term[k] = term_g[k];
	for (int k = threadIdx.x; k < num_tables; k += blockDim.x) {
		const Table t = tables_g[k];
		tabs[k] = SmemTable{t.start, t.step_inv, static_cast<int>(t.size),
							static_cast<int>(t.pot - values_g)};
	}
	for (uint32_t k = threadIdx.x; k < total_values; k += blockDim.x) vals[k] = values_g[k];
	__syncthreads();

	const int lane = threadIdx.x & (G - 1);
	const uint32_t groups = blockDim.x / G;
	const uint32_t i = blockIdx.x * groups + threadIdx.x / G;
	double e_acc = 0.0, w_acc = 0.0;
	// Rows past n get an empty range so that every lane reaches the group
	// reduction below (the shuffles need the whole warp).
	const bool valid = i < n;
	const float4 pi = valid ? sorted_pos[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	const uint32_t* trow = term + (valid ? type_of(pi) : 0) * T;
	float fx = 0.0f, fy = 0.0f, fz = 0.0f, fe = 0.0f;
	{
		const uint32_t beg = valid ? row_start[i] : 0u;
		const uint32_t end = valid ? row_start[i + 1] : 0u;
		for (uint32_t p = beg + lane; p < end; p += G) {
			const uint32_t entry = nbr[p];
			const uint32_t j = entry & ~kOrientBit;
			const float4 pj = sorted_pos[j];
			// Reference orientation: r = wrap_diff(pos[second] - pos[first]).
			float dx = __fsub_rn(pj.x, pi.x), dy = __fsub_rn(pj.y, pi.y),
				  dz = __fsub_rn(pj.z, pi.z);
			const uint32_t flip = entry & kOrientBit;
			dx = __uint_as_float(__float_as_uint(dx) ^ flip);
			dy = __uint_as_float(__float_as_uint(dy) ^ flip);
			dz = __uint_as_float(__float_as_uint(dz) ^ flip);
			const float3 r = wrap_diff(box, dx, dy, dz);
			const float dist = __fsqrt_rn(len2(r.x, r.y, r.z));
			if (dist < 1e-6f) continue;
			if (cutoff_sq > 0.0f && __fmul_rn(dist, dist) > cutoff_sq) continue;
			const uint32_t tag = trow[type_of(pj)];
			if (!(tag & kTermTabulated)) continue;
			const SmemTable t = tabs[tag >> kTableShift];
			const float2 fm_e = table_lookup(vals + t.offset, t.size, t.start, t.step_inv, 0, dist);
			const float inv = __frcp_rn(dist);
			// f = unit * F (force on the pair's second particle)
			float gx = __fmul_rn(__fmul_rn(inv, r.x), fm_e.x);
			float gy = __fmul_rn(__fmul_rn(inv, r.y), fm_e.x);
			float gz = __fmul_rn(__fmul_rn(inv, r.z), fm_e.x);
			if (get_energy) {
				e_acc += static_cast<double>(fm_e.y);
				w_acc += static_cast<double>(gx) * r.x + static_cast<double>(gy) * r.y +
						 static_cast<double>(gz) * r.z;
			}
			// j is the second particle unless the pair is stored flipped.
			gx = __uint_as_float(__float_as_uint(gx) ^ flip);
			gy = __uint_as_float(__float_as_uint(gy) ^ flip);
			gz = __uint_as_float(__float_as_uint(gz) ^ flip);
			const float half = get_energy ? __fmul_rn(fm_e.y, 0.5f) : 0.0f;
			red_add_v4(&force[j], gx, gy, gz, half);
			fx -= gx;
			fy -= gy;
			fz -= gz;
			fe += half;
		}
	}
#pragma unroll
	for (int o = G / 2; o > 0; o >>= 1) {
		fx += __shfl_xor_sync(0xFFFFFFFFu, fx, o, G);
		fy += __shfl_xor_sync(0xFFFFFFFFu, fy, o, G);
		fz += __shfl_xor_sync(0xFFFFFFFFu, fz, o, G);
		fe += __shfl_xor_sync(0xFFFFFFFFu, fe, o, G);
	}
	if (valid && lane == 0 && (fx != 0.0f || fy != 0.0f || fz != 0.0f || fe != 0.0f))
		red_add_v4(&force[i], fx, fy, fz, fe);
	if (get_energy) block_add_f64(e_acc, w_acc, ev);
}

__global__ void __launch_bounds__(256) scatter_add_kernel(const float4* __restrict__ fs,
														  const uint32_t* __restrict__ s2o,
														  uint32_t n, float4* __restrict__ fe,
														  int get_energy) {
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const float4 f = fs[s];
	const uint32_t o = s2o[s];
	float4 t = fe[o];
	t.x += f.x;
	t.y += f.y;
	t.z += f.z;
	if (get_energy) t.w += f.w;
	fe[o] = t;
}

// CalcDistance::compute (src/Interactions/Interactions.h:37-51).
__device__ __forceinline__ float calc_distance(const Box& box, const float4& from,
											   const float4& to, float3& r, float3& unit) {
	r = wrap_diff(box, __fsub_rn(to.x, from.x), __fsub_rn(to.y, from.y), __fsub_rn(to.z, from.z));
	const float dist = __fsqrt_rn(len2(r.x, r.y, r.z));
	if (dist > 1e-6f) {
		const float inv = __frcp_rn(dist);
		unit = make_float3(__fmul_rn(inv, r.x), __fmul_rn(inv, r.y), __fmul_rn(inv, r.z));
	} else {
		unit = make_float3(0.0f, 0.0f, 0.0f);
	}
	return dist;
}

__device__ __forceinline__ void add_v4(float4* p, float x, float y, float z, float w) {
	red_add_v4(p, x, y, z, w);
}

// TabulatedBondComputer::operator() (src/Interactions/Bonded/BondComputer.h:168-191).
__global__ void __launch_bounds__(256) bond_kernel(const int2* __restrict__ bonds,
												   const int* __restrict__ table_idx, uint32_t nb,
												   const float4* __restrict__ pos, float4* fe,
												   const Table* __restrict__ tables, Box box,
												   int get_energy, double* energy) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	double e_acc = 0.0;
	if (k < nb) {
		const int2 b = bonds[k];
		float3 r, u;
		const float dist = calc_distance(box, pos[b.x], pos[b.y], r, u);
		if (dist >= 1e-6f) {
			const Table t = tables[table_idx[k]];
			const float2 fm_e =
				table_lookup(t.pot, static_cast<int>(t.size), t.start, t.step_inv, 0, dist);
			const float fx = __fmul_rn(u.x, fm_e.x), fy = __fmul_rn(u.y, fm_e.x),
						fz = __fmul_rn(u.z, fm_e.x);
			const float half = get_energy ? __fmul_rn(fm_e.y, 0.5f) : 0.0f;
			add_v4(&fe[b.x], -fx, -fy, -fz, half);
			add_v4(&fe[b.y], fx, fy, fz, half);
			e_acc = get_energy ? static_cast<double>(fm_e.y) : 0.0;
		}
	}
	if (get_energy) block_add_f64(e_acc, 0.0, energy);
}

// TabulatedAngleComputer::operator() (BondComputer.h:236-268) with
// AngleGeometry::compute (src/Interactions/Bonded/BondGeometry.h:19-44).
// Angle tables wrap (src/Interactions/DeviceBondedInteraction.h:234).
__global__ void __launch_bounds__(256) angle_kernel(const int4* __restrict__ angles,
													const int* __restrict__ table_idx, uint32_t na,
													const float4* __restrict__ pos, float4* fe,
													const Table* __restrict__ tables, Box box,
													int get_energy, double* energy) {
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	double e_acc = 0.0;
	if (k < na) {
		const int4 a = angles[k];
		const float4 pi = pos[a.x], pj = pos[a.y], pk = pos[a.z];
		const float3 ab = wrap_diff(box, __fsub_rn(pj.x, pi.x), __fsub_rn(pj.y, pi.y),
									__fsub_rn(pj.z, pi.z));
		const float3 bc = wrap_diff(box, __fsub_rn(pk.x, pj.x), __fsub_rn(pk.y, pj.y),
									__fsub_rn(pk.z, pj.z));
		const float3 ac = wrap_diff(box, __fsub_rn(pk.x, pi.x), __fsub_rn(pk.y, pi.y),
									__fsub_rn(pk.z, pi.z));
		const float ab2 = len2(ab.x, ab.y, ab.z), bc2 = len2(bc.x, bc.y, bc.z),
					ac2 = len2(ac.x, ac.y, ac.z);
		float cs = __fdiv_rn(__fmul_rn(__fsub_rn(__fadd_rn(ab2, bc2), ac2), 0.5f),
							 __fmul_rn(__fsqrt_rn(ab2), __fsqrt_rn(bc2)));
		if (cs < -1.0f) cs = -1.0f;
		if (cs > 1.0f) cs = 1.0f;
		const float angle = acosf(cs);
		const float sn = __fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(cs, cs)));
		const Table t = tables[table_idx[k]];
		const float2 fm_e =
			table_lookup(t.pot, static_cast<int>(t.size), t.start, t.step_inv, 1, angle);
		const float sin_angle = sn > 1e-3f ? sn : 1e-3f;
		const float dudt = __fdiv_rn(-fm_e.x, sin_angle);
		const float inv_ab = __frcp_rn(__fsqrt_rn(ab2));
		const float inv_bc = __frcp_rn(__fsqrt_rn(bc2));
		const float s1 = __fmul_rn(dudt, inv_ab);
		const float c_ab = __fmul_rn(cs, inv_ab);
		const float s3 = -__fmul_rn(dudt, inv_bc);
		const float c_bc = __fmul_rn(cs, inv_bc);
		const float f1x = __fmul_rn(s1, __fadd_rn(__fmul_rn(ab.x, c_ab), __fmul_rn(bc.x, inv_bc)));
		const float f1y = __fmul_rn(s1, __fadd_rn(__fmul_rn(ab.y, c_ab), __fmul_rn(bc.y, inv_bc)));
		const float f1z = __fmul_rn(s1, __fadd_rn(__fmul_rn(ab.z, c_ab), __fmul_rn(bc.z, inv_bc)));
		const float f3x = __fmul_rn(s3, __fadd_rn(__fmul_rn(bc.x, c_bc), __fmul_rn(ab.x, inv_ab)));
		const float f3y = __fmul_rn(s3, __fadd_rn(__fmul_rn(bc.y, c_bc), __fmul_rn(ab.y, inv_ab)));
		const float f3z = __fmul_rn(s3, __fadd_rn(__fmul_rn(bc.z, c_bc), __fmul_rn(ab.z, inv_ab)));
		const float third = get_energy ? __fmul_rn(fm_e.y, 0.3333333432674408f) : 0.0f;
		add_v4(&fe[a.x], f1x, f1y, f1z, third);
		add_v4(&fe[a.y], -__fadd_rn(f1x, f3x), -__fadd_rn(f1y, f3y), -__fadd_rn(f1z, f3z), third);
		add_v4(&fe[a.z], f3x, f3y, f3z, third);
		e_acc = get_energy ? static_cast<double>(fm_e.y) : 0.0;
	}
	if (get_energy) block_add_f64(e_acc, 0.0, energy);
}

template <int G>
void launch_pair(const float4* sorted_pos, const uint32_t* row_start, const uint32_t* nbr,
				 uint32_t n, const PairTables& t, const Box& box, float cutoff_sq, int get_energy,
				 float4* force_sorted, double* ev, cudaStream_t st) {
	const size_t smem = static_cast<size_t>((t.num_types * t.num_types + 3) & ~3) * 4 +
						static_cast<size_t>(t.num_tables) * sizeof(SmemTable) +
						static_cast<size_t>(t.total_values) * 4;
	auto kern = pair_force_kernel<G>;
	if (smem > 48 * 1024)
		MB2_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
									  static_cast<int>(smem)));
	const uint32_t groups = 256 / G;
	const uint32_t blocks = (n + groups - 1) / groups;
	MB2_LAUNCH kern<<<blocks, 256, smem, st>>>(sorted_pos, row_start, nbr, n, t.term_matrix, t.num_types,
									t.tables, t.num_tables, t.values, t.total_values, box,
									cutoff_sq, get_energy, force_sorted, ev);
}

}  // namespace

void pair_forces(const float4* sorted_pos, const uint32_t* row_start, const uint32_t* nbr,
				 uint32_t n, const PairTables& t, const Box& box, float cutoff_sq, int get_energy,
				 float4* force_sorted, double* ev, int lanes_per_row, cudaStream_t st) {
	if (n == 0) return;
	switch (lanes_per_row) {
	case 4: launch_pair<4>(sorted_pos, row_start, nbr, n, t, box, cutoff_sq, get_energy, force_sorted, ev, st); break;
	case 8: launch_pair<8>(sorted_pos, row_start, nbr, n, t, box, cutoff_sq, get_energy, force_sorted, ev, st); break;
	case 16: launch_pair<16>(sorted_pos, row_start, nbr, n, t, box, cutoff_sq, get_energy, force_sorted, ev, st); break;
	default: launch_pair<32>(sorted_pos, row_start, nbr, n, t, box, cutoff_sq, get_energy, force_sorted, ev, st); break;
	}
}

void scatter_add_forces(const float4* force_sorted, const uint32_t* s2o, uint32_t n,
						float4* force_energy, int get_energy, cudaStream_t st) {
	if (n == 0) return;
	MB2_LAUNCH scatter_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(force_sorted, s2o, n, force_energy,
														get_energy);
}

void bond_forces(const int2* bonds, const int* table_idx, uint32_t nb, const float4* pos,
				 float4* fe, const Table* tables, const Box& box, int get_energy, double* energy,
				 cudaStream_t st) {
	if (nb == 0) return;
	MB2_LAUNCH bond_kernel<<<(nb + 255) / 256, 256, 0, st>>>(bonds, table_idx, nb, pos, fe, tables, box,
												  get_energy, energy);
}

void angle_forces(const int4* angles, const int* table_idx, uint32_t na, const float4* pos,
				  float4* fe, const Table* tables, const Box& box, int get_energy, double* energy,
				  cudaStream_t st) {
	if (na == 0) return;
	MB2_LAUNCH angle_kernel<<<(na + 255) / 256, 256, 0, st>>>(angles, table_idx, na, pos, fe, tables, box,
												   get_energy, energy);
}

}  // namespace mb2
