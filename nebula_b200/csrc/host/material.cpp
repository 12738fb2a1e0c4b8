// Material files and the table transforms of the reference's material
// constructors.
//
// `.nmat` carries the content of the reference's HDF5 material file
// (io/hdf5_file.h:27-177): quantity properties with units, float datasets
// with a unit and a dimension scale per axis.  The transforms applied on
// load are those of kieft_elastic::create (physics/kieft/elastic.h:120-166),
// full_penn::create (physics/full_penn.h:294-406), kieft_inelastic::create
// (physics/kieft/inelastic.h:215-331) and material(hdf5_file)
// (core/material.inl:13-18); the double/float evaluation order follows them
// (and units::quantity, common/units/quantity.h, where eV, nm and
// dimensionless are 1 and g is 6.2415e15), so the tables equal the
// reference's bit for bit.
#include "internal.hpp"

#include <cmath>
#include <cstring>
#include <fstream>
#include <algorithm>

namespace nbl {
namespace {

struct Scale { bool present = false; std::string unit; std::vector<double> v; };
struct Dataset { std::string unit; std::vector<uint64_t> dims; std::vector<Scale> scales; std::vector<float> data; };
struct File {
	std::map<std::string, std::pair<double, std::string>> props;
	std::map<std::string, Dataset> sets;
};

// HDF5 resolves "a/b" and "/a/b" to the same dataset (the reference asks
// for "ionization/binding_icdf" in kieft/inelastic.h:263).
std::string canonical(const std::string& name)
{
	size_t i = 0;
	while (i < name.size() && name[i] == '/') ++i;
	return name.substr(i);
}

File parse(const std::string& path)
{
	std::ifstream f(path, std::ios::binary);
	require(bool(f), "cannot open material file " + path, NBL_ERR_IO);
	std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
	size_t off = 0;
	auto need = [&](size_t n) { require(off + n <= b.size(), "truncated material file " + path, NBL_ERR_IO); };
	auto u32 = [&]() { need(4); uint32_t v; std::memcpy(&v, &b[off], 4); off += 4; return v; };
	auto u64 = [&]() { need(8); uint64_t v; std::memcpy(&v, &b[off], 8); off += 8; return v; };
	auto f64 = [&]() { need(8); double v; std::memcpy(&v, &b[off], 8); off += 8; return v; };
	auto str = [&]() { uint32_t n = u32(); need(n); std::string s(b.data() + off, n); off += n; return s; };
	need(8);
	require(std::memcmp(b.data(), "NBLMAT01", 8) == 0, path + ": not a material file", NBL_ERR_IO);
	off = 8;
	File out;
	const uint32_t np = u32();
	for (uint32_t i = 0; i < np; ++i) {
		std::string k = str();
		const double v = f64();
		out.props[k] = { v, str() };
	}
	const uint32_t nd = u32();
	for (uint32_t i = 0; i < nd; ++i) {
		Dataset d;
		std::string k = str();
		d.unit = str();
		const uint32_t rank = u32();
		require(rank >= 1 && rank <= 3, path + ": dataset rank must be 1..3", NBL_ERR_IO);
		for (uint32_t a = 0; a < rank; ++a) d.dims.push_back(u64());
		for (uint32_t a = 0; a < rank; ++a) {
			need(1);
			Scale s;
			s.present = b[off++] != 0;
			if (s.present) {
				s.unit = str();
				s.v.resize(d.dims[a]);
				need(8 * d.dims[a]);
				std::memcpy(s.v.data(), &b[off], 8 * d.dims[a]);
				off += 8 * d.dims[a];
			}
			d.scales.push_back(s);
		}
		size_t cnt = 1;
		for (auto x : d.dims) {
			require(x >= 2 && x < (1u << 24), path + ": table axis must have 2..2^24 points", NBL_ERR_IO);
			cnt *= x;
		}
		d.data.resize(cnt);
		need(4 * cnt);
		std::memcpy(d.data.data(), &b[off], 4 * cnt);
		off += 4 * cnt;
		out.sets[canonical(k)] = std::move(d);
	}
	return out;
}

// Unit strings of the material files (unit_system.h:16-36: base units are 1).
double unit_value(const std::string& u)
{
	if (u.empty() || u == "eV" || u == "nm" || u == "nm^-1" || u == "dimensionless")
		return 1.0;
	if (u == "g")
		return 6.2415e15;
	throw Error(NBL_ERR_IO, "unsupported unit '" + u + "'");
}

// geomspace (range.h:264-327): first value and the recomputed last value.
void log_range(const Scale& s, double& first, double& last)
{
	require(s.present && s.v.size() >= 2, "logarithmic dimension scale missing", NBL_ERR_IO);
	const double u = unit_value(s.unit);
	const double a = s.v.front() * u, b = s.v.back() * u;
	const size_t n = s.v.size();
	const double step = std::log(b / a) / (n - 1);
	first = a;
	last = a * std::exp((n - 1) * step);
}
// linspace (range.h:204-262); an absent linear scale is [0, 1] (hdf5_file.cpp:298-300)
void lin_range(const Scale& s, size_t n, double& first, double& last)
{
	double a = 0, b = 1;
	if (s.present) {
		const double u = unit_value(s.unit);
		a = s.v.front() * u;
		b = s.v.back() * u;
	}
	const double step = (b - a) / (n - 1);
	first = a;
	last = a + (n - 1) * step;
}
// table set_scale: v_min = (float)lo, v_step = (n - 1) / (hi - lo) in float
void axis(int32_t n, double lo, double hi, bool log_axis, float& vmin, float& vstep)
{
	const float a = (float)(log_axis ? std::log(lo) : lo);
	const float b = (float)(log_axis ? std::log(hi) : hi);
	vmin = a;
	vstep = (n - 1) / (b - a);
}

// table_2D::get_rounddown (table_2D.inl:96-104) on the host
float rounddown2(const HostTable& t, float x, float y)
{
	const float xi = (x - t.x_min) * t.x_step;
	const float yi = (y - t.y_min) * t.y_step;
	const int ix = std::min(std::max((int)std::floor(xi), 0), t.nx - 1);
	const int iy = std::min(std::max((int)std::floor(yi), 0), t.ny - 1);
	return t.data[(size_t)ix * t.ny + iy];
}

// Ionisation table of the Kieft-Bosch model (kieft/inelastic.h:262-327):
// above 100 eV an inner shell from the binding ICDF at K + 10 eV (kept when
// >= 50 eV and finite), otherwise the largest outer shell (< 100 eV) not
// above K, otherwise -1.  The reference rewrites the table in place, row by
// row, while it reads it with get_rounddown, so later reads may see values
// already rewritten; the same order is kept here.
void load_kieft_binding(const std::string& path, Dataset& d, Dataset& shells, HostTable& t)
{
	double lo, hi;
	t.data = d.data;
	t.nx = (int32_t)d.dims[0]; t.ny = (int32_t)d.dims[1];
	log_range(d.scales[0], lo, hi); axis(t.nx, lo, hi, true, t.x_min, t.x_step);
	lin_range(d.scales[1], t.ny, lo, hi); axis(t.ny, lo, hi, false, t.y_min, t.y_step);
	std::vector<double> outer;
	{
		const double u = unit_value(shells.unit);
		for (float v : shells.data) {
			const double e = (double)v * u;
			if (e < 100)
				outer.push_back(e);
		}
		std::sort(outer.begin(), outer.end());
	}
	const double unit = unit_value(d.unit);
	const Scale& ks = d.scales[0];
	require(ks.present, path + ": binding_icdf energy scale missing", NBL_ERR_IO);
	const double ku = unit_value(ks.unit);
	const double kfirst = ks.v.front() * ku;
	const double kstep = std::log((ks.v.back() * ku) / kfirst) / (ks.v.size() - 1);
	double pfirst = 0, plast = 1;
	if (d.scales[1].present) {
		const double pu = unit_value(d.scales[1].unit);
		pfirst = d.scales[1].v.front() * pu;
		plast = d.scales[1].v.back() * pu;
	}
	const double pstep = (plast - pfirst) / (t.ny - 1);
	for (int32_t x = 0; x < t.nx; ++x) {
		const double K = kfirst * std::exp(x * kstep);
		for (int32_t y = 0; y < t.ny; ++y) {
			const float P = (float)(pfirst + y * pstep);
			const double margin = 10;
			double binding = -1;
			if (K > 100) {
				binding = (double)rounddown2(t, (float)std::log((K + margin) / 1.0), P) * unit;
				if (binding < 50 || !std::isfinite(binding))
					binding = -1;
			}
			if (binding < 0) {
				// largest outer shell <= K
				for (auto it = outer.rbegin(); it != outer.rend(); ++it)
					if (!(*it > K)) { binding = *it; break; }
			}
			t.data[(size_t)x * t.ny + y] = (float)(binding / 1.0);
		}
	}
}

}  // namespace

HostMaterial load_material_file(const std::string& path)
{
	File f = parse(path);
	auto prop = [&](const char* k) -> double {
		auto it = f.props.find(k);
		require(it != f.props.end(), path + ": missing property '" + k + "'", NBL_ERR_IO);
		return it->second.first * unit_value(it->second.second);
	};
	auto has = [&](const char* k) { return f.sets.count(canonical(k)) != 0; };
	auto set = [&](const char* k, size_t rank) -> Dataset& {
		auto it = f.sets.find(canonical(k));
		require(it != f.sets.end(), path + ": missing table '" + k + "'", NBL_ERR_IO);
		require(it->second.dims.size() == rank, path + ": table '" + k + "' has the wrong rank", NBL_ERR_IO);
		return it->second;
	};
	HostMaterial m;
	double lo, hi;

	const bool penn = has("/full_penn/imfp"), kieft = has("/inelastic_kieft/imfp");
	require(penn || kieft, path + ": no inelastic model tables (/full_penn or /inelastic_kieft)", NBL_ERR_IO);
	m.models = (penn ? 1 : 0) | (kieft ? 2 : 0);

	// inverse mean free paths: log(imfp * unit) (elastic.h:129-140,
	// full_penn.h:306-317, kieft/inelastic.h:226-238)
	auto imfp = [&](const char* name, HostTable& t) {
		Dataset& d = set(name, 1);
		t.data = d.data;
		const float unit = (float)(unit_value(d.unit) * 1.0);
		for (float& v : t.data)
			v = std::log(v * unit);
		t.nx = (int32_t)d.dims[0];
		log_range(d.scales[0], lo, hi);
		axis(t.nx, lo, hi, true, t.x_min, t.x_step);
	};
	imfp("/elastic/imfp", m.el_imfp);
	{	// cos(theta) ICDF clipped to [-1, 1] (elastic.h:144-157)
		Dataset& d = set("/elastic/costheta_icdf", 2);
		HostTable& t = m.el_icdf;
		t.data = d.data;
		for (float& v : t.data)
			v = std::max(-1.0f, std::min(1.0f, v));
		t.nx = (int32_t)d.dims[0]; t.ny = (int32_t)d.dims[1];
		log_range(d.scales[0], lo, hi); axis(t.nx, lo, hi, true, t.x_min, t.x_step);
		lin_range(d.scales[1], t.ny, lo, hi); axis(t.ny, lo, hi, false, t.y_min, t.y_step);
	}
	const double fermi_q = prop("fermi");
	// energy-loss ICDF: log(max(0, min(K - fermi, omega))) (full_penn.h:321-344,
	// kieft/inelastic.h:240-261)
	auto loss_icdf = [&](const char* name, HostTable& t) {
		Dataset& d = set(name, 2);
		t.data = d.data;
		const float unit = (float)(unit_value(d.unit) / 1.0);
		const Scale& ks = d.scales[0];
		require(ks.present, path + ": omega_icdf energy scale missing", NBL_ERR_IO);
		const double u = unit_value(ks.unit);
		const double first = ks.v.front() * u;
		const double step = std::log((ks.v.back() * u) / first) / (ks.v.size() - 1);
		for (size_t x = 0; x < d.dims[0]; ++x) {
			const double K = first * std::exp(x * step);
			for (size_t y = 0; y < d.dims[1]; ++y) {
				float& v = t.data[x * d.dims[1] + y];
				v = (float)std::log(std::max(0.0, std::min<double>((K - fermi_q) / 1.0, v * unit)));
			}
		}
		t.nx = (int32_t)d.dims[0]; t.ny = (int32_t)d.dims[1];
		log_range(d.scales[0], lo, hi); axis(t.nx, lo, hi, true, t.x_min, t.x_step);
		lin_range(d.scales[1], t.ny, lo, hi); axis(t.ny, lo, hi, false, t.y_min, t.y_step);
	};
	if (penn) {
	imfp("/full_penn/imfp", m.in_imfp);
	loss_icdf("/full_penn/omega_icdf", m.in_omega);
	{	// q ICDF in eV^1/2: q * hbar/sqrt(2m) (full_penn.h:348-369)
		Dataset& d = set("/full_penn/q_icdf", 3);
		HostTable& t = m.in_q;
		t.data = d.data;
		const float unit = (float)(unit_value(d.unit) * 0.19519 * 1.0);
		for (float& v : t.data)
			v = v * unit;
		t.nx = (int32_t)d.dims[0]; t.ny = (int32_t)d.dims[1]; t.nz = (int32_t)d.dims[2];
		log_range(d.scales[0], lo, hi); axis(t.nx, lo, hi, true, t.x_min, t.x_step);
		lin_range(d.scales[1], t.ny, lo, hi); axis(t.ny, lo, hi, false, t.y_min, t.y_step);
		lin_range(d.scales[2], t.nz, lo, hi); axis(t.nz, lo, hi, false, t.z_min, t.z_step);
	}
	{	// inner-shell binding ICDF, < 50 eV or non-finite -> -1 (full_penn.h:374-402)
		Dataset& d = set("/ionization/binding_icdf", 3);
		HostTable& t = m.in_binding;
		t.data = d.data;
		const float unit = (float)(unit_value(d.unit) / 1.0);
		for (float& v : t.data) {
			float b = v * unit;
			if (b < 50 || !std::isfinite(b))
				b = -1;
			v = b;
		}
		t.nx = (int32_t)d.dims[0]; t.ny = (int32_t)d.dims[1]; t.nz = (int32_t)d.dims[2];
		log_range(d.scales[0], lo, hi); axis(t.nx, lo, hi, true, t.x_min, t.x_step);
		log_range(d.scales[1], lo, hi); axis(t.ny, lo, hi, true, t.y_min, t.y_step);
		lin_range(d.scales[2], t.nz, lo, hi); axis(t.nz, lo, hi, false, t.z_min, t.z_step);
	}
	}
	if (kieft) {
		imfp("/inelastic_kieft/imfp", m.ki_imfp);
		loss_icdf("/inelastic_kieft/w0_icdf", m.ki_w0);
		load_kieft_binding(path, set("ionization/binding_icdf", 2), set("ionization/outer_shells", 1), m.ki_binding);
	}
	m.fermi = (float)(fermi_q / 1.0);
	{
		auto it = f.props.find("band_gap");
		m.band_gap = (float)((it == f.props.end() ? -1.0 : it->second.first * unit_value(it->second.second)) / 1.0);
	}
	m.barrier = (float)(prop("barrier") / 1.0);
	m.phonon_loss = (float)(prop("phonon_loss") / 1.0);
	m.recoil_const = 2 * (float)(((6.2415e15 * 9.109383e-28) * 2) / prop("effective_A"));
	return m;
}

}  // namespace nbl
