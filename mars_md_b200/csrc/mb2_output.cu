// Output side of the step: DCD trajectory frames, the energy file and
// restart files of one system, written as SimManager writes them
// (src/SimManager.cpp:596-633 write_dcd_frame, :833-861 the momentum DCD,
// :999-1068 write_energy_output, :1078-1135 write_restart_files) through a
// DCD writer with DcdWriter's byte layout (src/IO/DcdWriter.h).
//
// The reference copies every particle array to the host, un-permutes it by
// global id there (DeviceParticle::copy_to_host_unpermuted), and sums energies
// in host loops. Here one kernel scatters positions (and momenta and type ids)
// by global id straight into the X / Y / Z blocks a DCD frame stores, one
// asynchronous copy brings 12 bytes per particle per block set to pinned
// memory, and a writer thread puts them on disk while the next steps run.
// Energies are FP64 reductions on the device; only two doubles come back.
#include "../../include/marsb200.h"
#include "mb2_internal.cuh"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <charconv>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <deque>
#include <fstream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace mb2;

namespace {

constexpr float kSqrtCalToJoule = 2.046167337f;  // constants::SQRT_CAL_TO_JOULE

// Scatter by global id: block b (x, y, z of positions; then of momenta) of
// the staging area gets component b of row i at index ids[i]; type ids too.
// An id outside [0, n) sets *bad and is not written (the reference throws).
__global__ void __launch_bounds__(256) pack_kernel(const float4* __restrict__ pos,
												   const float4* __restrict__ mom,
												   const int* __restrict__ type_ids,
												   const int* __restrict__ ids, uint32_t n,
												   float* __restrict__ stage, int* bad) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int g = ids ? ids[i] : static_cast<int>(i);
	if (g < 0 || static_cast<uint32_t>(g) >= n) {
		atomicOr(bad, 1);
		return;
	}
	const size_t s = static_cast<size_t>(n);
	if (pos) {
		const float4 p = pos[i];
		stage[g] = p.x;
		stage[s + g] = p.y;
		stage[2 * s + g] = p.z;
	}
	if (mom) {
		const float4 m = mom[i];
		stage[3 * s + g] = m.x;
		stage[4 * s + g] = m.y;
		stage[5 * s + g] = m.z;
	}
	if (type_ids) reinterpret_cast<int*>(stage + 6 * s)[g] = type_ids[i];
}

__device__ __forceinline__ void block_sum2(double a, double b, double* out) {
	__shared__ double ra[32], rb[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int o = 16; o > 0; o >>= 1) {
		a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
		b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
	}
	if (lane == 0) {
		ra[warp] = a;
		rb[warp] = b;
	}
	__syncthreads();
	if (warp == 0) {
		const int nw = blockDim.x >> 5;
		a = lane < nw ? ra[lane] : 0.0;
		b = lane < nw ? rb[lane] : 0.0;
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

// out[0] += sum of the per-particle energies (ForceEnergy .w), out[1] += sum of
// 0.5 |p|^2 / m (write_energy_output, SimManager.cpp:1003-1023): |p|^2 in
// float as Vector3::length2 rounds it, the rest in double. Grid-stride.
__global__ void __launch_bounds__(256) energy_kernel(const float4* __restrict__ fe,
													 const float4* __restrict__ mom,
													 const int* __restrict__ type_ids,
													 const float* __restrict__ mass, uint32_t n,
													 double* out) {
	double pe = 0.0, ke = 0.0;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		if (fe) pe += static_cast<double>(fe[i].w);
		if (mom) {
			const float4 p = mom[i];
			const float l2 = __fadd_rn(__fadd_rn(__fmul_rn(p.x, p.x), __fmul_rn(p.y, p.y)),
									   __fmul_rn(p.z, p.z));
			ke += 0.5 * static_cast<double>(l2) / static_cast<double>(mass[type_ids[i]]);
		}
	}
	block_sum2(pe, ke, out);
}

// DCD file with DcdWriter's layout (src/IO/DcdWriter.h): an existing file is
// renamed to <name>.BAK; the 84-byte header block (CORD, NFILE, NPRIV, NSAVC,
// NSTEP, DELTA, unit-cell flag, CHARMM version 24), two 80-character title
// lines, the atom count; per frame an optional 48-byte unit cell and the X,
// Y, Z blocks, each in Fortran record markers; NFILE and NSTEP in the header
// advance by 1 and NSAVC per frame.
class DcdFile {
  public:
	~DcdFile() { close(); }
	void open(const std::string& path) {
		path_ = path;
		struct stat sb;
		if (stat(path.c_str(), &sb) == 0) {
			const std::string bak = path + ".BAK";
			if (rename(path.c_str(), bak.c_str()) != 0)
				throw Error{MB2_ERR_IO, "DCD: cannot move the existing " + path + " aside"};
		}
		fd_ = ::open(path.c_str(), O_RDWR | O_CREAT | O_EXCL, S_IRUSR | S_IWUSR | S_IRGRP | S_IROTH);
		if (fd_ < 0) throw Error{MB2_ERR_IO, "DCD: cannot create " + path};
	}
	void header(int n, int nsavc, float delta, bool unitcell) {
		nsavc_ = nsavc;
		nfile_ = 0;
		nstep_ = nsavc - nsavc;  // NPRIV - NSAVC with NPRIV = NSAVC
		std::vector<char> b;
		auto i32 = [&](int32_t v) { b.insert(b.end(), reinterpret_cast<char*>(&v), reinterpret_cast<char*>(&v) + 4); };
		auto f32 = [&](float v) { b.insert(b.end(), reinterpret_cast<char*>(&v), reinterpret_cast<char*>(&v) + 4); };
		i32(84);
		b.insert(b.end(), {'C', 'O', 'R', 'D'});
		i32(0);         // NFILE, advanced per frame
		i32(nsavc);     // NPRIV
		i32(nsavc);     // NSAVC
		i32(nstep_);    // NSTEP, advanced per frame
		for (int k = 0; k < 5; ++k) i32(0);
		f32(delta);
		i32(unitcell ? 1 : 0);
		for (int k = 0; k < 8; ++k) i32(0);
		i32(24);        // CHARMM version
		i32(84);
		i32(164);
		i32(2);
		char line[200];
		std::snprintf(line, sizeof(line), "REMARKS FILENAME=%s CREATED BY MARS2", path_.c_str());
		title(b, line);
		const time_t now = time(nullptr);
		char date[11];
		std::strftime(date, sizeof(date), "%m/%d/%y", localtime(&now));
		std::snprintf(line, sizeof(line), "REMARKS DATE: %s CREATED BY USER: MARS2", date);
		title(b, line);
		i32(164);
		i32(4);
		i32(n);
		i32(4);
		write_all(b.data(), b.size());
	}
	// blocks: X, Y, Z of n floats, contiguous.
	void frame(const float* xyz, int n, const double* cell) {
		std::vector<char> b;
		b.reserve(static_cast<size_t>(n) * 12 + 96);
		auto raw = [&](const void* p, size_t bytes) {
			b.insert(b.end(), static_cast<const char*>(p), static_cast<const char*>(p) + bytes);
		};
		if (cell) {
			const int32_t m = 48;
			raw(&m, 4);
			raw(cell, 48);
			raw(&m, 4);
		}
		const int32_t m = n * 4;
		for (int a = 0; a < 3; ++a) {
			raw(&m, 4);
			raw(xyz + static_cast<size_t>(a) * n, static_cast<size_t>(n) * 4);
			raw(&m, 4);
		}
		write_all(b.data(), b.size());
		nstep_ += nsavc_;
		nfile_ += 1;
		if (pwrite(fd_, &nstep_, 4, 20) != 4 || pwrite(fd_, &nfile_, 4, 8) != 4)
			throw Error{MB2_ERR_IO, "DCD: header update failed for " + path_};
	}
	void close() {
		if (fd_ >= 0) ::close(fd_);
		fd_ = -1;
	}

  private:
	static void title(std::vector<char>& b, const char* s) {
		char line[81];
		std::memset(line, ' ', 80);
		const size_t len = std::min<size_t>(std::strlen(s), 80);
		std::memcpy(line, s, len);
		b.insert(b.end(), line, line + 80);
	}
	void write_all(const char* p, size_t bytes) {
		while (bytes) {
			const ssize_t w = ::write(fd_, p, bytes);
			if (w <= 0) throw Error{MB2_ERR_IO, "DCD: write failed for " + path_};
			p += w;
			bytes -= static_cast<size_t>(w);
		}
	}
	std::string path_;
	int fd_ = -1;
	int32_t nsavc_ = 1, nfile_ = 0, nstep_ = 0;
};

// "type x y z\n" with the shortest round-trip decimal of each value
// (append_restart_line, SimManager.cpp:14-28, std::to_chars).
void restart_text(const float* xyz, const int* types, uint32_t n, std::string& buf) {
	buf.clear();
	buf.reserve(static_cast<size_t>(n) * 40);
	char tmp[64];
	const size_t s = n;
	for (uint32_t i = 0; i < n; ++i) {
		auto r = std::to_chars(tmp, tmp + sizeof(tmp), types[i]);
		buf.append(tmp, r.ptr);
		for (int a = 0; a < 3; ++a) {
			buf.push_back(' ');
			r = std::to_chars(tmp, tmp + sizeof(tmp), xyz[a * s + i]);
			buf.append(tmp, r.ptr);
		}
		buf.push_back('\n');
	}
}

void write_file(const std::string& path, const std::string& text) {
	FILE* f = std::fopen(path.c_str(), "w");
	if (!f) throw Error{MB2_ERR_IO, "cannot open " + path};
	const size_t w = std::fwrite(text.data(), 1, text.size(), f);
	std::fclose(f);
	if (w != text.size()) throw Error{MB2_ERR_IO, "short write to " + path};
}

}  // namespace

struct mb2_output {
	std::string name;
	uint32_t n = 0;
	int nsavc = 1;
	float delta = 1.0f;
	float box[3] = {0, 0, 0};
	bool unitcell = false;
	bool momentum = false;
	int device = 0;
	std::string last_error;

	float* stage = nullptr;  // device: 7 n words (pos xyz, mom xyz, type)
	int* bad = nullptr;      // device flag
	double* esum = nullptr;  // device: potential, kinetic
	DevBuf<float> mass;

	// Two pinned slots, each 7 n words + one flag word.
	struct Slot {
		float* host = nullptr;
		cudaEvent_t ready = nullptr;
		bool busy = false;
	};
	Slot slots[2];

	struct Job {
		int slot;
		int kind;  // 0 frame, 1 restart
	};
	std::thread writer;
	std::mutex mu;
	std::condition_variable cv_job, cv_slot;
	std::deque<Job> jobs;
	bool stop = false;
	int in_flight = 0;
	std::string async_error;

	DcdFile dcd, dcd_mom;
	bool header_written = false;
	std::ofstream energy_file;

	void run_writer() {
		cudaSetDevice(device);
		std::string text;
		for (;;) {
			Job job;
			{
				std::unique_lock<std::mutex> lk(mu);
				cv_job.wait(lk, [&] { return stop || !jobs.empty(); });
				if (jobs.empty()) return;
				job = jobs.front();
				jobs.pop_front();
			}
			Slot& s = slots[job.slot];
			std::string err;
			try {
				MB2_CUDA(cudaEventSynchronize(s.ready));
				const float* h = s.host;
				const int* flag = reinterpret_cast<const int*>(h + 7 * static_cast<size_t>(n));
				if (*flag) throw Error{MB2_ERR_ARG, "output: a global id lies outside [0, n)"};
				if (job.kind == 0) {
					const double cell[6] = {box[0], 0.0, box[1], 0.0, 0.0, box[2]};
					if (!header_written) {
						dcd.header(static_cast<int>(n), nsavc, delta, unitcell);
						if (momentum) dcd_mom.header(static_cast<int>(n), nsavc, delta, unitcell);
						header_written = true;
					}
					dcd.frame(h, static_cast<int>(n), unitcell ? cell : nullptr);
					if (momentum)
						dcd_mom.frame(h + 3 * static_cast<size_t>(n), static_cast<int>(n),
									  unitcell ? cell : nullptr);
				} else {
					const int* types = reinterpret_cast<const int*>(h + 6 * static_cast<size_t>(n));
					restart_text(h, types, n, text);
					write_file(name + ".restart", text);
					if (momentum) {
						restart_text(h + 3 * static_cast<size_t>(n), types, n, text);
						write_file(name + ".0.momentum.restart", text);
					}
				}
			} catch (const Error& e) {
				err = e.msg;
			} catch (const std::exception& e) {
				err = e.what();
			}
			{
				std::lock_guard<std::mutex> lk(mu);
				if (!err.empty() && async_error.empty()) async_error = err;
				s.busy = false;
				--in_flight;
			}
			cv_slot.notify_all();
		}
	}

	int acquire_slot() {
		std::unique_lock<std::mutex> lk(mu);
		cv_slot.wait(lk, [&] { return !slots[0].busy || !slots[1].busy; });
		const int k = slots[0].busy ? 1 : 0;
		slots[k].busy = true;
		++in_flight;
		return k;
	}

	void submit(int slot, int kind) {
		{
			std::lock_guard<std::mutex> lk(mu);
			jobs.push_back(Job{slot, kind});
		}
		cv_job.notify_one();
	}

	void release_unsubmitted(int slot) {
		{
			std::lock_guard<std::mutex> lk(mu);
			slots[slot].busy = false;
			--in_flight;
		}
		cv_slot.notify_all();
	}

	void raise_async_error() {
		std::lock_guard<std::mutex> lk(mu);
		if (!async_error.empty()) {
			std::string e = async_error;
			async_error.clear();
			throw Error{MB2_ERR_IO, e};
		}
	}

	// Pack on the device and queue the copy to a pinned slot; the writer
	// thread waits for it and writes.
	void stage_and_submit(const float* pos4, const float* mom4, const int* type_ids,
						  const int* ids, uint32_t count, int kind, cudaStream_t st) {
		expect_arg(count == n, MB2_ERR_ARG, "output: n differs from the configured particle count");
		raise_async_error();
		const int k = acquire_slot();
		try {
			MB2_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
			MB2_LAUNCH pack_kernel<<<(n + 255) / 256, 256, 0, st>>>(
				reinterpret_cast<const float4*>(pos4), reinterpret_cast<const float4*>(mom4),
				type_ids, ids, n, stage, bad);
			MB2_CUDA(cudaGetLastError());
			const size_t words = (kind == 0 ? (momentum ? 6 : 3) : 7) * static_cast<size_t>(n);
			MB2_CUDA(cudaMemcpyAsync(slots[k].host, stage, words * 4, cudaMemcpyDeviceToHost, st));
			MB2_CUDA(cudaMemcpyAsync(slots[k].host + 7 * static_cast<size_t>(n), bad, sizeof(int),
									 cudaMemcpyDeviceToHost, st));
			MB2_CUDA(cudaEventRecord(slots[k].ready, st));
		} catch (...) {
			release_unsubmitted(k);
			throw;
		}
		submit(k, kind);
	}

	void drain() {
		std::unique_lock<std::mutex> lk(mu);
		cv_slot.wait(lk, [&] { return in_flight == 0; });
	}

	void release() {
		{
			std::lock_guard<std::mutex> lk(mu);
			stop = true;
		}
		cv_job.notify_all();
		if (writer.joinable()) writer.join();
		for (Slot& s : slots) {
			if (s.host) cudaFreeHost(s.host);
			if (s.ready) cudaEventDestroy(s.ready);
		}
		if (stage) cudaFree(stage);
		if (bad) cudaFree(bad);
		if (esum) cudaFree(esum);
	}
};

namespace {

template <typename F>
int oguard(mb2_output* o, F&& f) {
	if (!o) return MB2_ERR_ARG;
	try {
		MB2_CUDA(cudaSetDevice(o->device));
		f();
		o->last_error.clear();
		return MB2_OK;
	} catch (const Error& e) {
		o->last_error = e.msg;
		return e.code;
	} catch (const std::exception& e) {
		o->last_error = e.what();
		return MB2_ERR_IO;
	}
}

}  // namespace

extern "C" {

int mb2_output_create(const mb2_output_config* cfg, mb2_output** out) {
	if (!cfg || !out || !cfg->output_name || cfg->num_particles == 0) return MB2_ERR_ARG;
	mb2_output* o = new mb2_output();
	o->name = cfg->output_name;
	o->n = cfg->num_particles;
	o->nsavc = cfg->output_period > 1 ? cfg->output_period : 1;
	o->delta = cfg->timestep;
	for (int a = 0; a < 3; ++a) o->box[a] = cfg->box[a];
	o->unitcell = cfg->periodic[0] || cfg->periodic[1] || cfg->periodic[2];
	o->momentum = cfg->with_momentum != 0;
	o->device = cfg->device;
	const int rc = oguard(o, [&] {
		const size_t words = 7 * static_cast<size_t>(o->n);
		MB2_CUDA(cudaMalloc(&o->stage, words * 4));
		MB2_CUDA(cudaMalloc(&o->bad, sizeof(int)));
		MB2_CUDA(cudaMalloc(&o->esum, 2 * sizeof(double)));
		for (auto& s : o->slots) {
			MB2_CUDA(cudaMallocHost(&s.host, (words + 1) * 4));
			MB2_CUDA(cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming));
		}
		o->dcd.open(o->name + ".dcd");
		if (o->momentum) o->dcd_mom.open(o->name + ".0.momentum.dcd");
		o->writer = std::thread([o] { o->run_writer(); });
	});
	if (rc != MB2_OK) {
		o->release();
		delete o;
		return rc;
	}
	*out = o;
	return MB2_OK;
}

int mb2_output_destroy(mb2_output* o) {
	if (!o) return MB2_ERR_ARG;
	o->drain();
	o->release();
	delete o;
	return MB2_OK;
}

const char* mb2_output_last_error(const mb2_output* o) {
	return o ? o->last_error.c_str() : "null output";
}

int mb2_output_frame(mb2_output* o, const float* pos4, const float* mom4, const int* ids,
					 uint32_t n, void* stream) {
	return oguard(o, [&] {
		expect_arg(pos4 != nullptr, MB2_ERR_ARG, "mb2_output_frame: null positions");
		expect_arg(!o->momentum || mom4, MB2_ERR_ARG,
				   "mb2_output_frame: this output writes momenta; pass them");
		o->stage_and_submit(pos4, o->momentum ? mom4 : nullptr, nullptr, ids, n, 0,
							reinterpret_cast<cudaStream_t>(stream));
	});
}

int mb2_output_restart(mb2_output* o, const float* pos4, const float* mom4, const int* type_ids,
					   const int* ids, uint32_t n, void* stream) {
	return oguard(o, [&] {
		expect_arg(pos4 && type_ids, MB2_ERR_ARG, "mb2_output_restart: null positions or types");
		expect_arg(!o->momentum || mom4, MB2_ERR_ARG,
				   "mb2_output_restart: this output writes momenta; pass them");
		o->stage_and_submit(pos4, o->momentum ? mom4 : nullptr, type_ids, ids, n, 1,
							reinterpret_cast<cudaStream_t>(stream));
	});
}

int mb2_output_energy(mb2_output* o, const float* fe4, const float* mom4, const int* type_ids,
					  const float* mass, int num_types, uint32_t n, float kT, void* stream,
					  double out[2]) {
	return oguard(o, [&] {
		expect_arg(fe4 != nullptr && n == o->n, MB2_ERR_ARG,
				   "mb2_output_energy: null force/energy or n differs");
		expect_arg(!mom4 || (type_ids && mass && num_types > 0), MB2_ERR_ARG,
				   "mb2_output_energy: momenta need type ids and per-type masses");
		const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
		if (mom4) {
			o->mass.ensure(num_types);
			MB2_CUDA(cudaMemcpyAsync(o->mass.ptr, mass, num_types * sizeof(float),
									 cudaMemcpyHostToDevice, st));
		}
		MB2_CUDA(cudaMemsetAsync(o->esum, 0, 2 * sizeof(double), st));
		const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, 148 * 8);
		MB2_LAUNCH energy_kernel<<<blocks, 256, 0, st>>>(
			reinterpret_cast<const float4*>(fe4), reinterpret_cast<const float4*>(mom4), type_ids,
			mom4 ? o->mass.ptr : nullptr, n, o->esum);
		MB2_CUDA(cudaGetLastError());
		double h[2];
		MB2_CUDA(cudaMemcpyAsync(h, o->esum, sizeof(h), cudaMemcpyDeviceToHost, st));
		MB2_CUDA(cudaStreamSynchronize(st));
		const double potential = h[0];
		const double kinetic_kcal = h[1] / (kSqrtCalToJoule * kSqrtCalToJoule);
		const double kinetic_kT = kT > 0.0f ? kinetic_kcal / kT : 0.0;
		if (!o->energy_file.is_open()) o->energy_file.open(o->name + ".energy.dat");
		if (!o->energy_file.is_open())
			throw Error{MB2_ERR_IO, "cannot open " + o->name + ".energy.dat"};
		o->energy_file << "Kinetic Energy: " << kinetic_kT << " (kT) " << std::endl;
		o->energy_file << "Potential Energy: " << potential << " (kcal/mol) " << std::endl;
		if (out) {
			out[0] = kinetic_kT;
			out[1] = potential;
		}
	});
}

int mb2_output_flush(mb2_output* o) {
	return oguard(o, [&] {
		o->drain();
		o->raise_async_error();
	});
}

}  // extern "C"
