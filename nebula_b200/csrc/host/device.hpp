// Device-side helpers shared by the host implementation files: status
// checks, owning device buffers, and the device copies of geometry and
// materials.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include <string>
#include <algorithm>
#include "internal.hpp"
#include "../kernels.cuh"

namespace nbl {

#define CU(call)                                                                          \
	do {                                                                                  \
		cudaError_t e_ = (call);                                                          \
		if (e_ != cudaSuccess)                                                            \
			throw Error(e_ == cudaErrorMemoryAllocation ? NBL_ERR_OOM : NBL_ERR_CUDA,     \
				std::string(#call) + ": " + cudaGetErrorString(e_));                     \
	} while (0)

inline void set_device(int device)
{
	int n = 0;
	if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
		throw Error(NBL_ERR_NO_DEVICE, "no CUDA device available");
	require(device >= 0 && device < n, "device ordinal out of range");
	CU(cudaSetDevice(device));
}

// Device buffer that frees itself.
struct DevBuf {
	void* p = nullptr;
	size_t bytes = 0;
	DevBuf() = default;
	explicit DevBuf(size_t n) { alloc(n); }
	void alloc(size_t n)
	{
		release();
		if (n == 0) return;
		CU(cudaMalloc(&p, n));
		bytes = n;
	}
	void release()
	{
		if (p) cudaFree(p);
		p = nullptr;
		bytes = 0;
	}
	~DevBuf() { release(); }
	DevBuf(const DevBuf&) = delete;
	DevBuf& operator=(const DevBuf&) = delete;
	template<class T> T* as() const { return static_cast<T*>(p); }
};

// Triangles in the 64-byte device layout; normal = cross(e1, e2) in float
// with the operations of triangle::get_normal (core/triangle.inl:75-78).
inline std::vector<DevTriangle> device_triangles(const std::vector<nbl_triangle>& tris)
{
	std::vector<DevTriangle> out(tris.size());
	for (size_t i = 0; i < tris.size(); ++i) {
		const nbl_triangle& t = tris[i];
		DevTriangle& d = out[i];
		d.r0x = t.r0[0]; d.r0y = t.r0[1]; d.r0z = t.r0[2]; d.mat_in = t.material_in;
		d.e1x = t.e1[0]; d.e1y = t.e1[1]; d.e1z = t.e1[2]; d.mat_out = t.material_out;
		d.e2x = t.e2[0]; d.e2y = t.e2[1]; d.e2z = t.e2[2]; d.pad0 = 0;
		const float* a = t.e1;
		const float* b = t.e2;
		d.nx = a[1] * b[2] - a[2] * b[1];
		d.ny = a[2] * b[0] - a[0] * b[2];
		d.nz = a[0] * b[1] - a[1] * b[0];
		d.pad1 = 0;
	}
	return out;
}

// Geometry resident on one device.
struct DeviceGeometry {
	DevBuf octree, tris;
	DevGeometry view{};
	void upload(const HostGeometry& g, cudaStream_t s)
	{
		const std::vector<DevTriangle> dt = device_triangles(g.tris);
		octree.alloc(g.octree.size() * sizeof(int32_t));
		tris.alloc(std::max<size_t>(dt.size(), 1) * sizeof(DevTriangle));
		CU(cudaMemcpyAsync(octree.p, g.octree.data(), g.octree.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
		if (!dt.empty())
			CU(cudaMemcpyAsync(tris.p, dt.data(), dt.size() * sizeof(DevTriangle), cudaMemcpyHostToDevice, s));
		CU(cudaStreamSynchronize(s));
		view.octree = octree.as<int32_t>();
		view.tris = tris.as<DevTriangle>();
		view.cx = g.center[0]; view.cy = g.center[1]; view.cz = g.center[2];
		view.hx = g.halfsize[0]; view.hy = g.halfsize[1]; view.hz = g.halfsize[2];
		view.max_extent = g.max_extent;
		view.n_tri = (int32_t)g.tris.size();
		view.n_octree = (int64_t)g.octree.size();
	}
};

// Materials resident on one device: one buffer of all tables plus the
// DevMaterial array pointing into it.
struct DeviceMaterials {
	DevBuf tables, mats;
	int n = 0;
	std::vector<DevMaterial> host;   // the device array's contents
	void upload(const std::vector<const HostMaterial*>& ms, cudaStream_t s, uint32_t phys = PH_DEFAULT)
	{
		const bool kieft = (phys & PH_KIEFT) != 0;
		n = (int)ms.size();
		std::vector<float> blob;
		std::vector<size_t> offs;
		auto add = [&](const HostTable& t) {
			size_t o = blob.size();
			o = (o + 31) & ~size_t(31);   // 128-byte aligned tables
			blob.resize(o);
			offs.push_back(o);
			blob.insert(blob.end(), t.data.begin(), t.data.end());
		};
		for (const HostMaterial* m : ms) {
			const InelasticTables it = inelastic_tables(*m, kieft);
			add(m->el_imfp); add(m->el_icdf); add(*it.imfp); add(*it.omega); add(*it.q); add(*it.binding);
		}
		tables.alloc(std::max<size_t>(blob.size(), 1) * sizeof(float));
		CU(cudaMemcpyAsync(tables.p, blob.data(), blob.size() * sizeof(float), cudaMemcpyHostToDevice, s));
		std::vector<DevMaterial> dm(ms.size());
		const float* base = tables.as<float>();
		size_t k = 0;
		auto dev = [&](const HostTable& t) {
			DevTable d;
			d.data = base + offs[k++];
			d.nx = t.nx; d.ny = t.ny; d.nz = t.nz; d.pad = 0;
			d.x_min = t.x_min; d.x_step = t.x_step; d.y_min = t.y_min; d.y_step = t.y_step;
			d.z_min = t.z_min; d.z_step = t.z_step;
			return d;
		};
		for (size_t i = 0; i < ms.size(); ++i) {
			const HostMaterial& m = *ms[i];
			DevMaterial& d = dm[i];
			const InelasticTables it = inelastic_tables(m, kieft);
			d.el_imfp = dev(m.el_imfp); d.el_icdf = dev(m.el_icdf); d.in_imfp = dev(*it.imfp);
			d.in_omega = dev(*it.omega); d.in_q = dev(*it.q); d.in_binding = dev(*it.binding);
			d.fermi = m.fermi; d.band_gap = m.band_gap; d.barrier = m.barrier;
			d.phonon_loss = m.phonon_loss; d.recoil_const = m.recoil_const;
			d.in_scale = 1.0f; d.el_scale = 1.0f; d.pad = 0;
		}
		mats.alloc(std::max<size_t>(dm.size(), 1) * sizeof(DevMaterial));
		CU(cudaMemcpyAsync(mats.p, dm.data(), dm.size() * sizeof(DevMaterial), cudaMemcpyHostToDevice, s));
		CU(cudaStreamSynchronize(s));
		host = dm;
	}
};

}  // namespace nbl
